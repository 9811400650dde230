// PageRank sweep over the row-slice layout (sm_100a): pagerank_onepart
// (pr.cpp:119-154) for a resident graph.
//
// Per record (v0, v1) of tile (i, j) the reference does
//     rank[v1] += prior[v0];   rank[v0] += prior[v1]   (the second: half grid)
// with an FP32 compare-and-swap add (qthread_dincr, pr.cpp:60-80).  Both ends
// are random inside their 65,536-vertex windows, and the float state of a
// window (x and s, 512 KB) does not fit in shared memory, so the first
// version sent four random 4-byte operations per record to L2/DRAM.
//
// Here each tile's records are grouped by row slice (v0 >> 13: eight slices
// of 8,192 vertices) in a second copy of the records, sorted by v1 inside a
// slice.  A CTA takes one work item — a row window, one slice, and the tiles
// of that row inside a block of kPrColBlock column windows — and
//   * stages x of the row slice (32 KB) in shared memory with one bulk copy,
//   * accumulates the row ends' sums in shared memory (32 KB),
//   * sends the column end's add to global memory (one `red` per record) and
//     reads x of the column end from global memory,
//   * flushes the row sums with 16-byte vector atomics.
// Items are ordered column block first, so the CTAs in flight share a few
// column blocks and the column ends' x and s stay in L2.  The sums are
// re-associated (row partial sums per item), which only changes float
// rounding.
#include "gs_internal.cuh"
#include "gs_ops.cuh"

#include <algorithm>
#include <vector>

namespace {

using namespace gsops;

constexpr int kPrThreads = 512;
constexpr int kPrWarps = kPrThreads / 32;
constexpr uint32_t kSliceVerts = 1u << kPrSliceBits;   // 8192
constexpr int kSlices = 1 << (kTileBits - kPrSliceBits);  // 8
constexpr long long kWaitLimit = 1ll << 24;

struct __align__(128) PrSmem {
    float xs[kSliceVerts];
    float ys[kSliceVerts];
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

struct PrSliceOp {
    const float* xs;     // shared: x of the row slice
    float* ys;           // shared: sums of the row slice
    const float* x;
    float* y;
    int directed;
    // Records of a slice are sorted by v1, so a lane meets the same column
    // end many times in a row on high-degree columns: it keeps the column
    // end's x and a running sum, and adds to y once per run of equal v1
    // (fewer atomics, and shorter FP32 accumulation chains).
    struct Item {
        uint32_t cb;
        uint32_t pb;     // column end of the open run, ~0 = none
        float xb;        // x[pb]
        float sum;       // sum of x[a] over the open run
    };
    __device__ bool begin(uint32_t, uint32_t col, Item& c) const {
        c.cb = col << 16;
        c.pb = ~0u;
        c.xb = 0.f;
        c.sum = 0.f;
        return true;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = r & (kSliceVerts - 1), b = c.cb + (r >> 16);
        const float xa = xs[a];
        if (b != c.pb) {
            if (c.pb != ~0u) atomicAdd(y + c.pb, c.sum);   // pr.cpp:145-146
            c.pb = b;
            c.sum = 0.f;
            if (!directed) c.xb = __ldg(x + b);
        }
        c.sum += xa;
        if (!directed) atomicAdd(ys + a, c.xb);            // pr.cpp:147-150
    }
    __device__ void end(uint32_t, uint32_t, Item& c) const {
        if (c.pb != ~0u) atomicAdd(y + c.pb, c.sum);
    }
};

__global__ void __launch_bounds__(kPrThreads, 2)
    pr_slice_kernel(const gs_pr_item* __restrict__ items, uint64_t n_items, const gs_unit* __restrict__ units,
                    const uint32_t* __restrict__ rec, const float* __restrict__ x, float* __restrict__ y,
                    int directed, int* error, unsigned int* ticket) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    PrSmem& m = *reinterpret_cast<PrSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&m.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const PrSliceOp op{m.xs, m.ys, x, y, directed};
    uint32_t parity = 0;
    // the next item from `ticket` when one is given, else every gridDim.x-th
    __shared__ unsigned long long s_item;
    auto advance = [&](uint64_t i) -> uint64_t {
        if (!ticket) return i + gridDim.x;
        __syncthreads();   // every thread has read the previous draw
        if (tid == 0) s_item = atomicAdd(ticket, 1u);
        __syncthreads();
        return s_item;
    };
    for (uint64_t i = ticket ? advance(0) : blockIdx.x; i < n_items; i = advance(i)) {
        const gs_pr_item it = items[i];
        const uint64_t base = ((uint64_t)it.row << kTileBits) + ((uint64_t)it.slice << kPrSliceBits);
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&m.bar)),
                         "r"(kSliceVerts * 4)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(m.xs)),
                "l"(x + base), "r"(kSliceVerts * 4), "r"(smem_u32(&m.bar))
                : "memory");
        }
        if (!directed)
            for (uint32_t k = tid; k < kSliceVerts; k += kPrThreads) m.ys[k] = 0.f;
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
        for (uint32_t ui = it.unit_beg + warp; ui < it.unit_end; ui += kPrWarps) sweep_unit(units[ui], rec, op, lane);
        __syncthreads();
        if (!directed) {
            const float4* s4 = reinterpret_cast<const float4*>(m.ys);
            float4* y4 = reinterpret_cast<float4*>(y + base);
            for (uint32_t k = tid; k < kSliceVerts / 4; k += kPrThreads) {
                const float4 v = s4[k];
                if (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f) atomicAdd(y4 + k, v);
            }
        }
        __syncthreads();   // xs and ys are rewritten by the next item
    }
    if (ticket && tid == 0 && atomicAdd(ticket + 1, 1u) == gridDim.x - 1) {
        atomicExch(ticket, 0u);   // every CTA has drawn its last ticket
        atomicExch(ticket + 1, 0u);
    }
}

// Record <-> slice-major key: (v0 >> 13) in bits 29-31, v1 in bits 13-28,
// v0 & 0x1FFF in bits 0-12, so a per-tile sort groups records by row slice
// and orders them by v1 inside it.
__global__ void to_slice_key(uint32_t* rec, uint64_t n) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = tid; k < n; k += nth) {
        const uint32_t r = rec[k], v0 = r & 0xFFFFu, v1 = r >> 16;
        rec[k] = ((v0 >> kPrSliceBits) << 29) | (v1 << kPrSliceBits) | (v0 & (kSliceVerts - 1));
    }
}

__global__ void from_slice_key(uint32_t* rec, uint64_t n) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = tid; k < n; k += nth) {
        const uint32_t key = rec[k];
        const uint32_t v0 = ((key >> 29) << kPrSliceBits) | (key & (kSliceVerts - 1));
        const uint32_t v1 = (key >> kPrSliceBits) & 0xFFFFu;
        rec[k] = v0 | (v1 << 16);
    }
}

// Per tile: where each row slice starts (keys sorted inside the tile).
__global__ void slice_bounds(const uint32_t* __restrict__ key, const uint64_t* __restrict__ tile_off, uint64_t T,
                             uint64_t* __restrict__ out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = tid; t < T; t += nth) {
        const uint64_t lo = tile_off[t], hi = tile_off[t + 1];
        out[t * kSlices] = lo;
        for (int s = 1; s < kSlices; ++s) {
            uint64_t a = lo, b = hi;   // first k with key[k] >> 29 >= s
            while (a < b) {
                const uint64_t mid = (a + b) >> 1;
                if ((key[mid] >> 29) < (uint32_t)s) a = mid + 1;
                else b = mid;
            }
            out[t * kSlices + s] = a;
        }
    }
}

inline uint32_t grid_for(uint64_t n, const gs_ctx* ctx) {
    const uint64_t b = (n + 255) / 256;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

}  // namespace

void pr_layout_free(gs_graph* g) {
    gs_dev_free(g->pr.d_rec);
    gs_dev_free(g->pr.d_units);
    gs_dev_free(g->pr.d_items);
    g->pr = gs_pr_layout();
}

gs_status pr_layout_build(gs_graph* g) {
    gs_ctx* ctx = g->ctx;
    gs_pr_layout& L = g->pr;
    const uint64_t E = g->E, T = g->T;
    pr_layout_free(g);
    GS_TRY(gs_alloc_records(ctx, &L.d_rec, E));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(L.d_rec, g->d_rec, E * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    to_slice_key<<<grid_for(E, ctx), 256, 0, ctx->stream>>>(L.d_rec, E);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_TRY(gs_sort_tiles(ctx, g->d_tile_off, T, L.d_rec, E));
    uint64_t* d_so = nullptr;
    GS_TRY(gs_dev_alloc(ctx, (void**)&d_so, std::max<uint64_t>(1, T) * kSlices * 8));
    slice_bounds<<<grid_for(T, ctx), 256, 0, ctx->stream>>>(L.d_rec, g->d_tile_off, T, d_so);
    from_slice_key<<<grid_for(E, ctx), 256, 0, ctx->stream>>>(L.d_rec, E);
    ctx->launches += 2;
    std::vector<uint64_t> so(T * kSlices);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && T)
        e = cudaMemcpyAsync(so.data(), d_so, T * kSlices * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    gs_dev_free(d_so);
    if (e != cudaSuccess) return gs_cuda_fail(ctx, e, "row-slice layout");

    // segments: consecutive tiles of one row inside one column block
    struct Seg {
        uint32_t row, cb;
        uint32_t t0, t1;
    };
    std::vector<Seg> segs;
    for (uint32_t t = 0; t < T; ++t) {
        const uint32_t rc = g->h_tile_rc[t], row = rc >> 16, cb = (rc & 0xFFFFu) / kPrColBlock;
        if (!segs.empty() && segs.back().row == row && segs.back().cb == cb && segs.back().t1 == t)
            segs.back().t1 = t + 1;
        else
            segs.push_back(Seg{row, cb, t, t + 1});
    }
    std::stable_sort(segs.begin(), segs.end(),
                     [](const Seg& a, const Seg& b) { return a.cb != b.cb ? a.cb < b.cb : a.row < b.row; });
    std::vector<gs_unit> units;
    std::vector<gs_pr_item> items;
    units.reserve(T * 2 + E / kUnitRecords);
    for (const Seg& sg : segs) {
        for (int s = 0; s < kSlices; ++s) {
            const uint32_t u0 = (uint32_t)units.size();
            for (uint32_t t = sg.t0; t < sg.t1; ++t) {
                const uint64_t b = so[(uint64_t)t * kSlices + s];
                const uint64_t e2 = s + 1 < kSlices ? so[(uint64_t)t * kSlices + s + 1] : g->h_tile_off[t + 1];
                for (uint64_t x = b; x < e2; x += kUnitRecords)
                    units.push_back(gs_unit{x, (uint32_t)std::min<uint64_t>(kUnitRecords, e2 - x), g->h_tile_rc[t]});
            }
            if (units.size() > u0) items.push_back(gs_pr_item{u0, (uint32_t)units.size(), sg.row, (uint32_t)s});
        }
    }
    L.n_units = units.size();
    L.n_items = items.size();
    GS_TRY(gs_dev_alloc(ctx, (void**)&L.d_units, std::max<size_t>(1, units.size()) * sizeof(gs_unit)));
    GS_TRY(gs_dev_alloc(ctx, (void**)&L.d_items, std::max<size_t>(1, items.size()) * sizeof(gs_pr_item)));
    if (!units.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(L.d_units, units.data(), units.size() * sizeof(gs_unit),
                                           cudaMemcpyHostToDevice, ctx->stream));
    if (!items.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(L.d_items, items.data(), items.size() * sizeof(gs_pr_item),
                                           cudaMemcpyHostToDevice, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    L.built = true;
    return GS_OK;
}

gs_status pr_slice_sweep(gs_graph* g, cudaStream_t stream, const float* x, float* y, int* error, bool item_ctas) {
    gs_ctx* ctx = g->ctx;
    const gs_pr_layout& L = g->pr;
    if (L.n_items == 0) return GS_OK;
    GS_CHECK_CUDA(ctx, gs_smem_limit_once<pr_slice_kernel>(ctx->device, (int)sizeof(PrSmem)));
    // persistent (two CTAs per SM walking the items) or one CTA per item, so
    // that a higher-priority stream's CTAs find free SMs between items
    const uint32_t grid = (uint32_t)std::min<uint64_t>(L.n_items, item_ctas ? 0x7FFFFFFFull : gs_grid_size(ctx, 3));
    // the persistent form runs on the context's stream only, which owns the
    // PageRank ticket; one CTA per item needs none
    unsigned int* ticket = item_ctas ? nullptr : ctx->d_ticket + 2;
    pr_slice_kernel<<<grid, kPrThreads, sizeof(PrSmem), stream>>>(L.d_items, L.n_items, L.d_units, L.d_rec, x, y,
                                                                  g->directed, error, ticket);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return GS_OK;
}

gs_status pr_slice_launch(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_error) {
        GS_TRY(gs_state_alloc(s, (void**)&s->d_error, sizeof(uint64_t)));
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_error, 0, sizeof(uint64_t), ctx->stream));
    }
    gs_timer_begin(ctx);
    GS_TRY(pr_slice_sweep(g, ctx->stream, s->d_x, s->d_y, (int*)s->d_error));
    // algorithmic bytes per iteration: 4E + 12V (records, x, s, inv)
    gs_timer_end(ctx, GS_ALGO_PAGERANK, 4 * g->E + 12 * g->V);
    return GS_OK;
}
