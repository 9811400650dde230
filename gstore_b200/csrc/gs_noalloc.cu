// gs_bfs_noalloc: a BFS entry point that allocates no memory.
//
// Why it exists: some callers of this library are not allowed to allocate
// device memory while they run queries.  A host framework that owns the GPU
// through its own memory pool (a caching allocator that has already reserved
// most of HBM) cannot let a library call cudaMalloc behind its back — the
// call can fail once the pool holds the memory, and it defeats the pool's
// accounting — and a latency-sensitive serving loop cannot afford the
// device-wide synchronisation that cudaMalloc / cudaFree imply.  For them,
// this entry point runs the same BFS sweep kernels as gs_run on a BFS state,
// but keeps the per-vertex scratch state (frontier/visited bits, discovery
// bits, window flags, counters) in one array that is part of the library
// image, and writes the result into a buffer the caller already owns.
//
// Rules that follow from that design:
//   * the graph must have at most kNoAllocMaxVertices vertices (one tile
//     group, 2^24); larger graphs are rejected with GS_ERR_RANGE;
//   * the scratch array takes about 6 MiB on every GPU that loads the
//     library, for as long as the process lives;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) and remembers it; make that first call before
//     any stream capture on the device;
//   * every call uses the same array: calls that overlap on the GPU (on
//     different streams, threads or contexts of one device) race and give
//     wrong results; run them one after another.  Each call clears the parts
//     of the array it reads before using them.
#include "gs_internal.cuh"

#include <mutex>

namespace {

constexpr uint64_t kNoAllocMaxVertices = 1ull << 24;
constexpr uint64_t kNoAllocWindows = kNoAllocMaxVertices >> 16;

// Layout of the scratch array.
constexpr size_t kStOff = 0;                                              // 2-bit state, N/4 bytes
constexpr size_t kNextOff = kStOff + kNoAllocMaxVertices / 4;            // discovery bits, N/8 bytes
constexpr size_t kActOff = kNextOff + kNoAllocMaxVertices / 8;           // window flags
constexpr size_t kActNextOff = kActOff + kNoAllocWindows;
constexpr size_t kCountOff = kActNextOff + kNoAllocWindows;              // level count (u64)
constexpr size_t kErrorOff = kCountOff + 8;                              // error flag (int)
constexpr size_t kTicketOff = kErrorOff + 8;                             // sweep run ticket (2 x u32)
constexpr size_t kScratchBytes = kTicketOff + 8;

static __device__ __align__(256) unsigned char g_bfs_scratch[kScratchBytes];

std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[256] = {nullptr};   // per device, looked up once

}  // namespace

extern "C" gs_status gs_bfs_noalloc(gs_graph* g, uint64_t root, uint8_t* d_depth, int64_t* levels_out) {
    if (!g || !d_depth) return GS_ERR_ARG;
    gs_ctx* ctx = g->ctx;
    if (g->N > kNoAllocMaxVertices)
        return gs_fail(ctx, GS_ERR_RANGE,
                       "gs_bfs_noalloc handles at most 16777216 vertices (its scratch array is fixed); "
                       "use gs_state_create/gs_run for larger graphs");
    if (root >= g->V) return gs_fail(ctx, GS_ERR_ARG, "BFS root out of range");
    if (g->stream) return gs_fail(ctx, GS_ERR_UNSUPPORTED, "gs_bfs_noalloc needs a graph resident in HBM");
    if (ctx->device < 0 || ctx->device >= 256) return gs_fail(ctx, GS_ERR_ARG, "device ordinal out of range");
    GS_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (!g_scratch_addr[ctx->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_bfs_scratch);
            if (e != cudaSuccess) return gs_cuda_fail(ctx, e, "cudaGetSymbolAddress(bfs scratch)");
            g_scratch_addr[ctx->device] = static_cast<unsigned char*>(p);
        }
        base = g_scratch_addr[ctx->device];
    }
    uint32_t* st = reinterpret_cast<uint32_t*>(base + kStOff);
    uint32_t* next = reinterpret_cast<uint32_t*>(base + kNextOff);
    uint8_t* act = base + kActOff;
    uint8_t* act_next = base + kActNextOff;
    unsigned long long* count = reinterpret_cast<unsigned long long*>(base + kCountOff);
    int* error = reinterpret_cast<int*>(base + kErrorOff);
    unsigned int* ticket = reinterpret_cast<unsigned int*>(base + kTicketOff);

    // the array keeps the previous call's contents: clear what this call reads
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(st, 0, g->N / 4, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(next, 0, g->N / 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(act, 0, 2 * kNoAllocWindows + 16, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(ticket, 0, 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(d_depth, 0, g->V, ctx->stream));   // INFTY = 0
    GS_TRY(bfs_seed_into(ctx, d_depth, st, act, root));
    uint8_t level = 1;
    int64_t sweeps = 0;
    while (true) {
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(count, 0, 8, ctx->stream));
        GS_TRY(bfs_level_into(ctx, g, d_depth, st, next, act, act_next, count, error, ticket, (uint8_t)(level + 1)));
        ++sweeps;
        // swap(read_part, read_part_next); read_part_next->reset()
        std::swap(act, act_next);
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(act_next, 0, kNoAllocWindows, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, count, 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars + 1, error, 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (ctx->h_scalars[1] != 0) return gs_fail(ctx, GS_ERR_TIMEOUT, "BFS sweep: a bounded wait gave up");
        if (ctx->h_scalars[0] == 0) break;
        if (level == 254) return gs_fail(ctx, GS_ERR_RANGE, "BFS exceeds 254 levels (u8 depth_t)");
        ++level;
    }
    if (levels_out) *levels_out = sweeps;
    return GS_OK;
}
