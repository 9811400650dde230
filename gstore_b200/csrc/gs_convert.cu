// In-memory converter "-c 1" on the device (grid::pre_grid + grid::proc_grid,
// gstore.cpp:1245-1458): edge pairs -> .start offsets, .grid records and
// .degree counts, as a resident graph.
//
//  1. count:   per non-self-loop edge, order (min, max) for the half grid,
//              find its tile, count it, count both endpoint degrees
//              (out-degree only for the directed grid) — gstore.cpp:1270-1312
//  2. scan:    exclusive prefix sum of the tile counts -> .start (:1316-1324)
//  3. scatter: each edge takes the next slot of its tile (:1403-1447)
//  4. sort:    records inside each tile are sorted by value (v1, then v0).
//              The reference leaves them in thread order, so any in-tile
//              order is a valid .grid; a sorted one is deterministic and lets
//              a warp's consecutive records touch neighbouring state words.
#include "gs_internal.cuh"

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

namespace {

__device__ __forceinline__ uint64_t dev_calc_index_half(uint64_t i, uint64_t j, uint64_t pc) {
    return ((i * ((pc << 1) - i - 1)) >> 1) + j;
}

// .start index of the tile holding (a, b), a <= b for the half grid.
__device__ __forceinline__ uint64_t tile_of(uint64_t a, uint64_t b, uint64_t p, int directed) {
    const uint64_t gi = a >> kGroupBits, gj = b >> kGroupBits;
    const uint64_t si = (a >> kTileBits) & 255, sj = (b >> kTileBits) & 255;
    if (directed) return ((gi * p + gj) << 16) + si * 256 + sj;
    if (gi == gj)
        return ((dev_calc_index_half(gi, gi, p) - gi) << 16) + ((gi * 257) << 7) +
               dev_calc_index_half(si, sj, 256);
    return ((dev_calc_index_half(gi, gj, p) - gi - 1) << 16) + (((gi + 1) * 257) << 7) + si * 256 + sj;
}

__global__ void count_kernel(const uint2* __restrict__ pairs, uint64_t n, uint64_t V, uint64_t p,
                             int directed, unsigned long long* __restrict__ counts, int32_t* __restrict__ deg,
                             int* bad) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = tid; k < n; k += nth) {
        const uint2 e = pairs[k];
        if (e.x == e.y) continue;  // is_self_loop
        if (e.x >= V || e.y >= V) {
            *bad = 1;
            continue;
        }
        uint64_t a = e.x, b = e.y;
        if (!directed && a > b) {
            a = e.y;
            b = e.x;
        }
        atomicAdd(counts + tile_of(a, b, p, directed), 1ull);
        atomicAdd(deg + e.x, 1);
        if (!directed) atomicAdd(deg + e.y, 1);
    }
}

__global__ void scatter_kernel(const uint2* __restrict__ pairs, uint64_t n, uint64_t p, int directed,
                               const uint64_t* __restrict__ start, unsigned int* __restrict__ cursor,
                               uint32_t* __restrict__ rec) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = tid; k < n; k += nth) {
        const uint2 e = pairs[k];
        if (e.x == e.y) continue;
        uint64_t a = e.x, b = e.y;
        if (!directed && a > b) {
            a = e.y;
            b = e.x;
        }
        const uint64_t t = tile_of(a, b, p, directed);
        const unsigned slot = atomicAdd(cursor + t, 1u);
        rec[start[t] + slot] = (uint32_t)(a & 0xFFFF) | ((uint32_t)(b & 0xFFFF) << 16);
    }
}

__global__ void rebase_offsets_kernel(const uint64_t* __restrict__ start, uint64_t t0, uint64_t n,
                                      int* __restrict__ out) {
    const uint64_t base = start[t0];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (int)(start[t0 + i] - base);
}

// Flags a tile whose records are not in ascending order (a warp per unit;
// a unit's first record is compared with the last one of the previous unit
// when both lie in the same tile).
__global__ void tiles_unsorted_kernel(const gs_unit* __restrict__ units, uint64_t n_units,
                                      const uint32_t* __restrict__ rec, int* flag) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = warp; u < n_units; u += n_warps) {
        const gs_unit un = units[u];
        const bool joined = u > 0 && units[u - 1].rc == un.rc && units[u - 1].rec_beg + units[u - 1].n == un.rec_beg;
        bool bad = false;
        for (uint32_t k = lane; k < un.n; k += 32) {
            const uint64_t e = un.rec_beg + k;
            if ((k > 0 || joined) && rec[e] < rec[e - 1]) bad = true;
        }
        if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicExch(flag, 1);
    }
}

}  // namespace

gs_status gs_order_tiles(gs_graph* g, bool* sorted_now) {
    gs_ctx* ctx = g->ctx;
    *sorted_now = false;
    if (!g->d_rec || g->E < 2 || g->U == 0) return GS_OK;
    int* d_flag = (int*)ctx->d_scalars;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream));
    tiles_unsorted_kernel<<<gs_grid_size(ctx, 8), 256, 0, ctx->stream>>>(g->d_units, g->U, g->d_rec, d_flag);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    int h_flag = 0;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!h_flag) return GS_OK;
    GS_TRY(gs_sort_tiles(ctx, g->d_tile_off, g->T, g->d_rec, g->E));
    *sorted_now = true;
    return GS_OK;
}

// Sorts the records of every tile in place (segments = tiles of `start`).
gs_status gs_sort_tiles(gs_ctx* ctx, const uint64_t* d_start, uint64_t n_tiles, uint32_t* d_rec, uint64_t n_rec) {
    if (n_rec < 2 || n_tiles == 0) return GS_OK;
    std::vector<uint64_t> h(n_tiles + 1);
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(h.data(), d_start, (n_tiles + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // chunks of whole tiles with at most 2^30 records and 2^24 tiles each
    const uint64_t kMaxRec = 1ull << 30, kMaxTiles = 1ull << 24;
    uint32_t* d_out = nullptr;
    int* d_off = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    gs_status st = gs_alloc_records(ctx, &d_out, n_rec);
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_off, (std::min(n_tiles, kMaxTiles) + 1) * sizeof(int));
    uint64_t t0 = 0;
    while (st == GS_OK && t0 < n_tiles) {
        uint64_t t1 = t0;
        while (t1 < n_tiles && t1 - t0 < kMaxTiles && h[t1 + 1] - h[t0] <= kMaxRec) ++t1;
        if (t1 == t0) {
            st = gs_fail(ctx, GS_ERR_FORMAT, "a tile holds more than 2^30 records");
            break;
        }
        const uint64_t nr = h[t1] - h[t0];
        if (nr > 1) {
            rebase_offsets_kernel<<<256, 256, 0, ctx->stream>>>(d_start, t0, t1 - t0, d_off);
            ctx->launches++;
            size_t need = 0;
            cudaError_t e = cub::DeviceSegmentedSort::SortKeys(nullptr, need, d_rec + h[t0], d_out + h[t0], (int)nr,
                                                               (int)(t1 - t0), d_off, d_off + 1, ctx->stream);
            if (e == cudaSuccess && need > tmp_bytes) {
                gs_dev_free(d_tmp);
                d_tmp = nullptr;
                tmp_bytes = need;
                st = gs_dev_alloc(ctx, &d_tmp, tmp_bytes);
            }
            if (e == cudaSuccess && st == GS_OK)
                e = cub::DeviceSegmentedSort::SortKeys(d_tmp, need, d_rec + h[t0], d_out + h[t0], (int)nr,
                                                       (int)(t1 - t0), d_off, d_off + 1, ctx->stream);
            if (e != cudaSuccess && st == GS_OK) st = gs_cuda_fail(ctx, e, "segmented sort");
            ctx->launches++;
        } else if (nr == 1) {
            cudaError_t e = cudaMemcpyAsync(d_out + h[t0], d_rec + h[t0], 4, cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "copy");
        }
        t0 = t1;
    }
    if (st == GS_OK) {
        cudaError_t e = cudaMemcpyAsync(d_rec, d_out, n_rec * 4, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "copy sorted records");
    } else {
        cudaStreamSynchronize(ctx->stream);
    }
    gs_dev_free(d_out);
    gs_dev_free(d_off);
    gs_dev_free(d_tmp);
    return st;
}

gs_status gs_convert_launch(gs_ctx* ctx, const uint32_t* d_pairs, uint64_t n_pairs, uint64_t V, int directed,
                            uint64_t** d_start_out, uint32_t** d_grid_out, int32_t** d_degree_out,
                            uint64_t* n_start, uint64_t* n_rec) {
    uint32_t p, ps;
    uint64_t T;
    gs_geometry_of(V, directed, &p, &ps, &T);
    uint64_t* d_start = nullptr;
    unsigned int* d_cursor = nullptr;
    int32_t* d_deg = nullptr;
    uint32_t* d_rec = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    int* d_bad = (int*)ctx->d_scalars;
    gs_status st = GS_OK;
    const uint2* pairs = reinterpret_cast<const uint2*>(d_pairs);
    const uint32_t blocks = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>((n_pairs + 255) / 256, gs_grid_size(ctx, 16)));
    uint64_t total = 0;
    int bad = 0;
#define CV_CHECK(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) {                         \
            st = gs_cuda_fail(ctx, e_, #call);           \
            goto fail;                                   \
        }                                                \
    } while (0)
    if ((st = gs_dev_alloc(ctx, (void**)&d_start, (T + 1) * 8)) != GS_OK) goto fail;
    if ((st = gs_dev_alloc(ctx, (void**)&d_deg, std::max<uint64_t>(V, 1) * 4)) != GS_OK) goto fail;
    CV_CHECK(cudaMemsetAsync(d_start, 0, (T + 1) * 8, ctx->stream));
    CV_CHECK(cudaMemsetAsync(d_deg, 0, V * 4, ctx->stream));
    CV_CHECK(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
    if (n_pairs) {
        count_kernel<<<blocks, 256, 0, ctx->stream>>>(pairs, n_pairs, V, p, directed,
                                                      (unsigned long long*)d_start, d_deg, d_bad);
        CV_CHECK(cudaGetLastError());
        ctx->launches++;
    }
    CV_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_start, d_start, T + 1, ctx->stream));
    if ((st = gs_dev_alloc(ctx, &d_tmp, tmp_bytes)) != GS_OK) goto fail;
    CV_CHECK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_start, d_start, T + 1, ctx->stream));
    CV_CHECK(cudaMemcpyAsync(&total, d_start + T, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CV_CHECK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CV_CHECK(cudaStreamSynchronize(ctx->stream));
    if (bad) {
        st = gs_fail(ctx, GS_ERR_FORMAT, "an edge endpoint is >= the vertex count");
        goto fail;
    }
    if ((st = gs_alloc_records(ctx, &d_rec, total)) != GS_OK) goto fail;
    if ((st = gs_dev_alloc(ctx, (void**)&d_cursor, T * 4)) != GS_OK) goto fail;
    CV_CHECK(cudaMemsetAsync(d_cursor, 0, T * 4, ctx->stream));
    if (n_pairs) {
        scatter_kernel<<<blocks, 256, 0, ctx->stream>>>(pairs, n_pairs, p, directed, d_start, d_cursor, d_rec);
        CV_CHECK(cudaGetLastError());
        ctx->launches++;
    }
    CV_CHECK(cudaStreamSynchronize(ctx->stream));
    gs_dev_free(d_cursor);
    d_cursor = nullptr;
    if ((st = gs_sort_tiles(ctx, d_start, T, d_rec, total)) != GS_OK) goto fail;
    gs_dev_free(d_tmp);
    *d_start_out = d_start;
    *d_grid_out = d_rec;
    *d_degree_out = d_deg;
    *n_start = T + 1;
    *n_rec = total;
    return GS_OK;
fail:
#undef CV_CHECK
    cudaStreamSynchronize(ctx->stream);
    gs_dev_free(d_start);
    gs_dev_free(d_cursor);
    gs_dev_free(d_deg);
    gs_dev_free(d_rec);
    gs_dev_free(d_tmp);
    return st;
}

extern "C" gs_status gs_convert(gs_ctx* ctx, const uint32_t* pairs, uint64_t n_pairs, int is_device,
                                uint64_t V, gs_graph** out) {
    if (!ctx || !out || (n_pairs && !pairs) || V == 0 || V > (1ull << 32)) return GS_ERR_ARG;
    *out = nullptr;
    const uint32_t* d_pairs = pairs;
    uint32_t* d_copy = nullptr;
    if (!is_device && n_pairs) {
        GS_TRY(gs_dev_alloc(ctx, (void**)&d_copy, n_pairs * 8));
        cudaError_t e = cudaMemcpyAsync(d_copy, pairs, n_pairs * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) {
            gs_dev_free(d_copy);
            return gs_cuda_fail(ctx, e, "copy pairs");
        }
        d_pairs = d_copy;
    }
    uint64_t* d_start = nullptr;
    uint32_t* d_rec = nullptr;
    int32_t* d_deg = nullptr;
    uint64_t n_start = 0, n_rec = 0;
    gs_status st = gs_convert_launch(ctx, d_pairs, n_pairs, V, ctx->directed, &d_start, &d_rec, &d_deg,
                                     &n_start, &n_rec);
    gs_dev_free(d_copy);
    if (st != GS_OK) return st;
    st = gs_graph_adopt(ctx, V, d_start, n_start, d_rec, n_rec, d_deg, out);
    gs_dev_free(d_start);
    gs_dev_free(d_deg);
    return st;
}
