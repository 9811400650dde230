// Graph500 Kronecker generator on the device, byte-identical to the
// generator vendored with the reference (graph500-generator/).
//
// Published algorithm restated here (Graph500 reference generator v2):
//  * PRNG: the order-5 multiple recursive generator of L'Ecuyer, Blouin and
//    Couture (1993), modulus 2^31-1: z_new = 107374182 z1 + 104480 z5
//    (splittable_mrg.c:18-35, mrg_orig_step :165-173).
//  * Edge ei draws from the stream started at position ei * 2^64
//    (graph_generator.c:190-195, mrg_skip(…, 0, ei, 0)).  The skip is a
//    product of powers of the 5x5 companion matrix; the tables of powers are
//    computed here at first use by repeated squaring, not read from the
//    reference's precomputed table.
//  * Each of the logN levels draws a quadrant with probabilities
//    A=.57, B=C=.19, D=.05 (graph_generator.c:26-68), with clip-and-flip on
//    the diagonal (:141-148), and the endpoints are scrambled by two
//    multiply/bit-reverse rounds keyed by two 64-bit values drawn at stream
//    position 50*2^128 + 7*2^64 (:120-130, :176-186).
//  * Seeds: make_mrg_seed (utils.c:48-55).
#include "gs_internal.cuh"

#include <mutex>

namespace {

constexpr uint32_t kM = 0x7FFFFFFFu;          // 2^31 - 1
constexpr uint32_t kX = 107374182u, kY = 104480u;
constexpr int kSkipBytes = 5;                 // edge indices below 2^40

struct Mat5 {
    uint32_t m[5][5];
};

__host__ __device__ inline uint32_t mod_reduce(uint64_t x) {
    // x < 2^63; Mersenne reduction for 2^31 - 1
    x = (x & kM) + (x >> 31);
    x = (x & kM) + (x >> 31);
    uint32_t t = (uint32_t)x;
    return t >= kM ? t - kM : t;
}

__host__ __device__ inline uint32_t mod_mul(uint32_t a, uint32_t b) { return mod_reduce((uint64_t)a * b); }

Mat5 mat_identity() {
    Mat5 r{};
    for (int i = 0; i < 5; ++i) r.m[i][i] = 1;
    return r;
}

Mat5 mat_companion() {
    Mat5 r{};
    r.m[0][0] = kX;
    r.m[0][4] = kY;
    for (int i = 1; i < 5; ++i) r.m[i][i - 1] = 1;
    return r;
}

Mat5 mat_mul(const Mat5& a, const Mat5& b) {
    Mat5 r{};
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) {
            uint64_t s = 0;
            for (int k = 0; k < 5; ++k) s += mod_mul(a.m[i][k], b.m[k][j]);
            r.m[i][j] = mod_reduce(s);
        }
    return r;
}

Mat5 mat_pow(Mat5 base, uint64_t e) {
    Mat5 r = mat_identity();
    while (e) {
        if (e & 1) r = mat_mul(r, base);
        base = mat_mul(base, base);
        e >>= 1;
    }
    return r;
}

void mat_apply(const Mat5& a, uint32_t z[5]) {
    uint32_t o[5];
    for (int i = 0; i < 5; ++i) {
        uint64_t s = 0;
        for (int k = 0; k < 5; ++k) s += mod_mul(a.m[i][k], z[k]);
        o[i] = mod_reduce(s);
    }
    for (int i = 0; i < 5; ++i) z[i] = o[i];
}

__host__ __device__ inline uint32_t mrg_next(uint32_t z[5]) {
    const uint32_t n = mod_reduce((uint64_t)kX * z[0] + (uint64_t)kY * z[4]);
    z[4] = z[3];
    z[3] = z[2];
    z[2] = z[1];
    z[1] = z[0];
    z[0] = n;
    return n;
}

// Tables: skip[k][v] = (A^(2^64))^(v * 256^k).
struct SkipTables {
    Mat5 skip[kSkipBytes][256];
};

std::mutex g_tables_mu;
SkipTables* g_host_tables = nullptr;

const SkipTables* host_tables() {
    std::lock_guard<std::mutex> lk(g_tables_mu);
    if (g_host_tables) return g_host_tables;
    SkipTables* t = new SkipTables();
    Mat5 step = mat_companion();
    for (int i = 0; i < 64; ++i) step = mat_mul(step, step);  // A^(2^64)
    for (int k = 0; k < kSkipBytes; ++k) {
        t->skip[k][0] = mat_identity();
        for (int v = 1; v < 256; ++v) t->skip[k][v] = mat_mul(t->skip[k][v - 1], step);
        for (int i = 0; i < 8; ++i) step = mat_mul(step, step);  // ^256
    }
    g_host_tables = t;
    return t;
}

__host__ __device__ inline uint32_t tab_load(const uint32_t* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

__host__ __device__ inline void apply_tab(const Mat5* __restrict__ a, uint32_t z[5]) {
    uint32_t o[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 5; ++k) s += mod_mul(tab_load(&a->m[i][k]), z[k]);
        o[i] = mod_reduce(s);
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) z[i] = o[i];
}

// graph_generator.c:41-68 with SPK_NOISE_LEVEL == 0.
__host__ __device__ inline int four_way(uint32_t z[5]) {
    const uint32_t limit = 0xFFFFFFFFu % 10000u;
    uint32_t val = mrg_next(z);
    while (val < limit) val = mrg_next(z);
    val %= 10000u;
    if (val < 1900u) return 1;
    val -= 1900u;
    if (val < 1900u) return 2;
    val -= 1900u;
    if (val < 5700u) return 0;
    return 3;
}

__host__ __device__ inline uint64_t bit_reverse64(uint64_t v) {
#ifdef __CUDA_ARCH__
    return __brevll(v);
#else
    uint64_t r = 0;
    for (int i = 0; i < 64; ++i) r |= ((v >> i) & 1ull) << (63 - i);
    return r;
#endif
}

__host__ __device__ inline uint64_t scramble(uint64_t v, int lgN, uint64_t val0, uint64_t val1) {
    v += val0 + val1;
    v *= (val0 | 0x4519840211493211ull);
    v = bit_reverse64(v) >> (64 - lgN);
    v *= (val1 | 0x3050852102C843A5ull);
    v = bit_reverse64(v) >> (64 - lgN);
    return v;
}

// One edge of the stream (make_one_edge, graph_generator.c:133-160).
__host__ __device__ inline void make_edge(const SkipTables* __restrict__ tab, const uint32_t seed[5], int lgN,
                                          uint64_t val0, uint64_t val1, uint64_t ei, uint32_t out[2]) {
    uint32_t z[5] = {seed[0], seed[1], seed[2], seed[3], seed[4]};
#pragma unroll 1
    for (int k = 0; k < kSkipBytes; ++k) {
        const uint32_t b = (uint32_t)(ei >> (8 * k)) & 0xFFu;
        if (b) apply_tab(&tab->skip[k][b], z);
    }
    uint64_t nverts = 1ull << lgN, bs = 0, bt = 0;
    while (nverts > 1) {
        const int sq = four_way(z);
        int so = sq / 2, to = sq % 2;
        if (bs == bt && so > to) {  // clip-and-flip
            const int tmp = so;
            so = to;
            to = tmp;
        }
        nverts >>= 1;
        bs += nverts * so;
        bt += nverts * to;
    }
    out[0] = (uint32_t)scramble(bs, lgN, val0, val1);
    out[1] = (uint32_t)scramble(bt, lgN, val0, val1);
}

__global__ void kron_kernel(const SkipTables* __restrict__ tab, uint32_t s0, uint32_t s1, uint32_t s2,
                            uint32_t s3, uint32_t s4, int lgN, uint64_t M, uint64_t val0, uint64_t val1,
                            uint2* __restrict__ out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const uint32_t seed[5] = {s0, s1, s2, s3, s4};
    for (uint64_t ei = tid; ei < M; ei += nth) {
        uint32_t e[2];
        make_edge(tab, seed, lgN, val0, val1, ei, e);
        out[ei] = make_uint2(e[0], e[1]);
    }
}

// Seeds (make_mrg_seed, utils.c:48-55) and the two scramble keys drawn at
// stream position 50 * 2^128 + 7 * 2^64 (graph_generator.c:176-186).
void kron_keys(uint64_t s1, uint64_t s2, uint32_t seed[5], uint64_t* val0, uint64_t* val1) {
    seed[0] = (uint32_t)((s1 & 0x3FFFFFFF) + 1);
    seed[1] = (uint32_t)(((s1 >> 30) & 0x3FFFFFFF) + 1);
    seed[2] = (uint32_t)((s2 & 0x3FFFFFFF) + 1);
    seed[3] = (uint32_t)(((s2 >> 30) & 0x3FFFFFFF) + 1);
    seed[4] = (uint32_t)(((s2 >> 60) << 4) + (s1 >> 60) + 1);
    uint32_t z[5] = {seed[0], seed[1], seed[2], seed[3], seed[4]};
    Mat5 b64 = mat_companion();
    for (int i = 0; i < 64; ++i) b64 = mat_mul(b64, b64);
    Mat5 b128 = b64;
    for (int i = 0; i < 64; ++i) b128 = mat_mul(b128, b128);
    mat_apply(mat_mul(mat_pow(b128, 50), mat_pow(b64, 7)), z);
    uint64_t v0 = mrg_next(z);
    v0 *= 0xFFFFFFFFull;
    v0 += mrg_next(z);
    uint64_t v1 = mrg_next(z);
    v1 *= 0xFFFFFFFFull;
    v1 += mrg_next(z);
    *val0 = v0;
    *val1 = v1;
}

struct DevTables {
    int device = -1;
    SkipTables* ptr = nullptr;
};
DevTables g_dev_tables[64];

}  // namespace

gs_status gs_kron_gen_launch(gs_ctx* ctx, int scale, int64_t ef, uint64_t s1, uint64_t s2,
                             uint32_t* d_pairs) {
    if (scale < 1 || scale > 32 || ef < 1) return gs_fail(ctx, GS_ERR_ARG, "bad scale/edgefactor");
    const uint64_t M = (uint64_t)ef << scale;
    if (M >= (1ull << (8 * kSkipBytes))) return gs_fail(ctx, GS_ERR_ARG, "too many edges");
    const SkipTables* ht = host_tables();
    SkipTables*& dt = g_dev_tables[ctx->device & 63].ptr;
    if (!dt) {
        GS_TRY(gs_dev_alloc(ctx, (void**)&dt, sizeof(SkipTables)));
        GS_CHECK_CUDA(ctx, cudaMemcpy(dt, ht, sizeof(SkipTables), cudaMemcpyHostToDevice));
    }
    uint32_t seed[5];
    uint64_t val0, val1;
    kron_keys(s1, s2, seed, &val0, &val1);
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((M + 255) / 256, gs_grid_size(ctx, 32));
    kron_kernel<<<blocks, 256, 0, ctx->stream>>>(dt, seed[0], seed[1], seed[2], seed[3], seed[4], scale, M,
                                                  val0, val1, reinterpret_cast<uint2*>(d_pairs));
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return GS_OK;
}

extern "C" {

gs_status gs_kron_generate_device(gs_ctx* ctx, int scale, int64_t edgefactor, uint64_t seed1,
                                  uint64_t seed2, uint32_t* d_pairs) {
    if (!ctx || !d_pairs) return GS_ERR_ARG;
    GS_TRY(gs_kron_gen_launch(ctx, scale, edgefactor, seed1, seed2, d_pairs));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

gs_status gs_kron_generate(gs_ctx* ctx, int scale, int64_t edgefactor, uint64_t seed1, uint64_t seed2,
                           uint32_t* host_pairs) {
    if (!ctx || !host_pairs || scale < 1 || scale > 32 || edgefactor < 1) return GS_ERR_ARG;
    const uint64_t M = (uint64_t)edgefactor << scale;
    uint32_t* d = nullptr;
    GS_TRY(gs_dev_alloc(ctx, (void**)&d, M * 8));
    gs_status st = gs_kron_gen_launch(ctx, scale, edgefactor, seed1, seed2, d);
    if (st == GS_OK) {
        cudaError_t e = cudaMemcpyAsync(host_pairs, d, M * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "copy edges");
    }
    gs_dev_free(d);
    return st;
}

}  // extern "C"
