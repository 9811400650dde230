// Per-record operations of the tile sweeps (sm_100a device code), shared by
// the per-algorithm sweep kernels and the batched persistent kernels.
//
// Reference semantics per record (edge_t{v0, v1} in tile (i, j)):
//   PR      pr.cpp:119-154      s[v1] += x[v0]; s[v0] += x[v1] (half grid)
//   WCC     wcc.cpp:177-278     hook the larger root onto the smaller one
//   k-core  kcore.cpp:63-177    --deg[other] for every removed endpoint
#pragma once

#include "gs_internal.cuh"

namespace gsops {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t bit_of(const uint32_t* __restrict__ bm, uint32_t v) {
    return (__ldg(bm + (v >> 5)) >> (v & 31)) & 1u;
}

__device__ __forceinline__ uint4 load_stream(const uint4* p) { return __ldcs(p); }

// One unit (<= kUnitRecords records of one tile) swept by one warp: the
// records stream with 128-bit evict-first loads from base (file record r at
// base[r]).  Op provides:
//   struct Item;                                    per-unit warp-uniform context
//   bool begin(uint32_t row, uint32_t col, Item&)   false = skip the unit
//   void record(uint32_t rec, Item&)                one record, any lane
//   void end(uint32_t row, uint32_t col, Item&)     warp-collective epilogue
template <class Op>
__device__ __forceinline__ void sweep_unit(const gs_unit d, const uint32_t* __restrict__ base, const Op& op,
                                           uint32_t lane) {
    const uint32_t row = d.rc >> 16, col = d.rc & 0xFFFFu;
    typename Op::Item ic;
    if (!op.begin(row, col, ic)) return;
    const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
    uint64_t ab = (b + 3) & ~3ull;
    if (ab > e) ab = e;
    uint64_t ae = e & ~3ull;
    if (ae < ab) ae = ab;
    if (b + lane < ab) op.record(__ldcs(base + b + lane), ic);
    if (ae + lane < e) op.record(__ldcs(base + ae + lane), ic);
    const uint4* r4 = reinterpret_cast<const uint4*>(base + ab);
    const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
    for (uint32_t k = lane; k < n4; k += 2 * 32) {
        const uint4 q0 = load_stream(r4 + k);
        const bool two = k + 32 < n4;
        uint4 q1 = make_uint4(0, 0, 0, 0);
        if (two) q1 = load_stream(r4 + k + 32);
        op.record(q0.x, ic);
        op.record(q0.y, ic);
        op.record(q0.z, ic);
        op.record(q0.w, ic);
        if (two) {
            op.record(q1.x, ic);
            op.record(q1.y, ic);
            op.record(q1.z, ic);
            op.record(q1.w, ic);
        }
    }
    op.end(row, col, ic);
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, (unsigned long long)v);
}

// --------------------------------------------------------------- PageRank --
// Acc: the type of the sums in y.  The sweep of a streamed graph adds in
// double: its per-record atomics reach high-degree vertices in file order,
// one add per record, and FP32 sums drift past the 1e-6 tolerance at
// Kronecker scale 28; that sweep waits on PCIe, so the wider adds cost no
// time.  x stays FP32.
template <class Acc>
struct PrOp {
    const float* x;
    Acc* y;
    int directed;
    // Tiles sorted by v1 (the device converter's order) give runs of equal
    // column ends per lane: one add to y per run (fewer atomics, shorter
    // FP32 accumulation chains); any order stays correct.
    struct Item {
        uint32_t rb, cb;
        uint32_t pb;     // column end of the open run, ~0 = none
        Acc xb;          // x[pb]
        Acc sum;         // sum of x[a] over the open run
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = row << 16;
        c.cb = col << 16;
        c.pb = ~0u;
        c.xb = 0;
        c.sum = 0;
        return true;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (b != c.pb) {
            if (c.pb != ~0u) atomicAdd(y + c.pb, c.sum);   // pr.cpp:145-146
            c.pb = b;
            c.sum = 0;
            if (!directed) c.xb = (Acc)__ldg(x + b);
        }
        c.sum += (Acc)__ldg(x + a);
        if (!directed) atomicAdd(y + a, c.xb);             // pr.cpp:147-150
    }
    __device__ void end(uint32_t, uint32_t, Item& c) const {
        if (c.pb != ~0u) atomicAdd(y + c.pb, c.sum);
    }
};

// -------------------------------------------------------------------- WCC --
__device__ __forceinline__ uint32_t find_root(const uint32_t* parent, uint32_t v) {
    uint32_t p = __ldcg(parent + v);
    while (p != v) {
        v = p;
        p = __ldcg(parent + v);
    }
    return v;
}

// find_root for kernels during which no tree is linked, so that roots stay
// roots: `known` is a root this thread found before, and a vertex pointing at
// it needs no second load.  After pointer jumping nearly every vertex of the
// largest tree points at one root, whose own entry every warp of the grid
// would otherwise read from a single L2 slice.  *first = parent[v].
__device__ __forceinline__ uint32_t find_root_known(const uint32_t* parent, uint32_t v, uint32_t& known,
                                                    uint32_t* first) {
    uint32_t p = __ldcg(parent + v);
    *first = p;
    if (p == v || p == known) return p;
    while (true) {
        const uint32_t pp = __ldcg(parent + p);
        if (pp == p) break;
        p = pp;
    }
    known = p;
    return p;
}

// find_root with path halving: every vertex passed on the way points to its
// grandparent afterwards.  Only non-roots are written (a vertex that has a
// parent never becomes a root again), always with one of their ancestors,
// so the stores never undo a link; without them the hooking sweeps build
// long parent chains and spend their time chasing them.
__device__ __forceinline__ uint32_t find_root_halving(uint32_t* parent, uint32_t v) {
    while (true) {
        const uint32_t p = __ldcg(parent + v);
        if (p == v) return v;
        const uint32_t gp = __ldcg(parent + p);
        if (gp == p) return p;
        __stcg(parent + v, gp);
        v = gp;
    }
}

// Links the trees of a and b (wcc.cpp:218-231, 263-275: toward the smaller
// id).  The larger root is linked under the smaller one with a
// compare-and-swap that succeeds only while it is still a root; when another
// record linked it first, the roots are found again.  No link is ever lost,
// so once a sweep has passed every record each record's ends share a root.
// Returns false only if the retries ran out (the record is left to the next
// sweep): every failed swap is another record's successful link, so this
// needs more than kHookRetries links to land on the same two trees while
// one record is being resolved.
constexpr int kHookRetries = 1 << 12;
__device__ __forceinline__ bool hook(uint32_t* parent, uint32_t a, uint32_t b) {
    uint32_t ra = find_root_halving(parent, a), rb = find_root_halving(parent, b);
    for (int i = 0; i < kHookRetries; ++i) {
        if (ra == rb) return true;
        const uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
        if (atomicCAS(parent + hi, hi, lo) == hi) return true;
        ra = find_root_halving(parent, hi);
        rb = find_root_halving(parent, lo);
    }
    return false;
}

// After the hooking sweeps: marks every vertex that some record joined to
// another -- every vertex whose parent is not itself, and every parent of
// such a vertex -- as touched (the label kernels give the others
// invalid_cid).  Hooking only ever links the trees of a record's two ends,
// so a vertex no record names keeps itself as parent and has no child.
static __global__ void wcc_mark_touched(const uint32_t* __restrict__ parent, uint8_t* touched, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint32_t last = ~0u;   // the parent marked last by this thread
    for (uint64_t v = tid; v < N; v += nth) {
        const uint32_t p = __ldcg(parent + v);
        if (p == v) continue;
        touched[v] = 1;
        if (p == last) continue;
        if (!touched[p]) touched[p] = 1;   // read first: a component's root is every member's parent
        last = p;
    }
}

struct WccOp {
    uint32_t* parent;
    uint8_t* touched;  // non-null on the first sweep
    unsigned long long* changes;   // records the sweep left unresolved (zero: the forest is final); may be null
    // Optional bitmap of vertices already known to share one tree (the
    // largest tree after a sampled hooking pass): a record with both ends in
    // it joins nothing new and is skipped without a parent lookup.
    const uint32_t* giant = nullptr;
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
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        // wcc.cpp:203-217: every record's ends get a label.  A record with two
        // ends joins them into one tree, which wcc_mark_touched finds after
        // the sweeps (a vertex with a parent, or with a child); only a
        // self-loop leaves its end alone in its tree, so only it is marked here
        if (touched && a == b) touched[a] = 1;
        if (giant && (bit_of(giant, a) & bit_of(giant, b))) return;
        // ends with one parent are in one tree (after pointer jumping most
        // vertices point at their root): two loads instead of four
        if (__ldcg(parent + a) == __ldcg(parent + b)) return;
        if (!hook(parent, a, b)) c.n += 1;
    }
    __device__ void end(uint32_t, uint32_t, Item& c) const {
        if (changes) warp_add_u64(changes, c.n);
    }
};

// ----------------------------------------------------------------- k-core --
struct KcoreOp {
    int32_t* deg;
    const uint32_t* removed;
    const uint8_t* act;
    struct Item {
        uint32_t rb, cb;
        bool fr, fc;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        // kcore_mmap dispatch (gstore.cpp:2773-2782)
        c.fr = act[row] != 0;
        c.fc = act[col] != 0;
        c.rb = row << 16;
        c.cb = col << 16;
        return c.fr || c.fc;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (c.fr && bit_of(removed, a)) atomicSub(deg + b, 1);  // kcore.cpp:77-78
        if (c.fc && bit_of(removed, b)) atomicSub(deg + a, 1);  // kcore.cpp:90-91
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

// ----------------------------------------------- multi-source BFS words --
// Per vertex {frontier, visited} words of a multi-source BFS, one bit per
// query (W = 32 or 64 queries).
template <class W>
struct FvPair;
template <>
struct alignas(8) FvPair<uint32_t> {
    uint32_t f, vis;
};
template <>
struct alignas(16) FvPair<unsigned long long> {
    unsigned long long f, vis;
};

__device__ __forceinline__ FvPair<uint32_t> load_fv(const FvPair<uint32_t>* p) {
    const uint2 x = __ldcg(reinterpret_cast<const uint2*>(p));
    return FvPair<uint32_t>{x.x, x.y};
}
__device__ __forceinline__ FvPair<unsigned long long> load_fv(const FvPair<unsigned long long>* p) {
    const ulonglong2 x = __ldcg(reinterpret_cast<const ulonglong2*>(p));
    return FvPair<unsigned long long>{x.x, x.y};
}
__device__ __forceinline__ void store_fv(FvPair<uint32_t>* p, uint32_t f, uint32_t vis) {
    __stcg(reinterpret_cast<uint2*>(p), make_uint2(f, vis));
}
__device__ __forceinline__ void store_fv(FvPair<unsigned long long>* p, unsigned long long f,
                                         unsigned long long vis) {
    ulonglong2 x;
    x.x = f;
    x.y = vis;
    __stcg(reinterpret_cast<ulonglong2*>(p), x);
}
__device__ __forceinline__ int popc_w(uint32_t x) { return __popc(x); }
__device__ __forceinline__ int popc_w(unsigned long long x) { return __popcll(x); }
template <class W>
__device__ __forceinline__ W warp_or(W x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(kFull, x, o);
    return x;
}
__device__ __forceinline__ int ffs_w(uint32_t x) { return __ffs(x); }
__device__ __forceinline__ int ffs_w(unsigned long long x) { return __ffsll((long long)x); }

// Multi-source sweep of one unit: per record (v0, v1), for all queries of
// the W-bit words at once, next[v1] |= f[v0] & ~vis[v1] and (half grid)
// next[v0] |= f[v1] & ~vis[v0] (bfs.cpp:158-172).  The {frontier, visited}
// pairs of a lane's four records are loaded before any of them is acted on,
// so eight loads are in flight at once.
template <class W>
__device__ __forceinline__ void ms_sweep_unit(const gs_unit d, const uint32_t* __restrict__ base, FvPair<W>* fv,
                                              W* next, int directed, uint32_t lane) {
    const uint32_t rb = (d.rc >> 16) << 16, cb = (d.rc & 0xFFFFu) << 16;
    auto act = [&](uint32_t a, uint32_t b, const FvPair<W>& sa, const FvPair<W>& sb) {
        const W nb = sa.f & ~sb.vis;
        if (nb) atomicOr(next + b, nb);
        if (!directed) {            // the half grid stores each edge once
            const W na = sb.f & ~sa.vis;
            if (na) atomicOr(next + a, na);
        }
    };
    auto one = [&](uint32_t r) {
        const uint32_t a = rb + (r & 0xFFFFu), b = cb + (r >> 16);
        act(a, b, load_fv(fv + a), load_fv(fv + b));
    };
    const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
    uint64_t ab = (b + 3) & ~3ull;
    if (ab > e) ab = e;
    uint64_t ae = e & ~3ull;
    if (ae < ab) ae = ab;
    if (b + lane < ab) one(__ldcs(base + b + lane));
    if (ae + lane < e) one(__ldcs(base + ae + lane));
    const uint4* r4 = reinterpret_cast<const uint4*>(base + ab);
    const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
    for (uint32_t k = lane; k < n4; k += 32) {
        const uint4 q = load_stream(r4 + k);
        const uint32_t a0 = rb + (q.x & 0xFFFFu), b0 = cb + (q.x >> 16);
        const uint32_t a1 = rb + (q.y & 0xFFFFu), b1 = cb + (q.y >> 16);
        const uint32_t a2 = rb + (q.z & 0xFFFFu), b2 = cb + (q.z >> 16);
        const uint32_t a3 = rb + (q.w & 0xFFFFu), b3 = cb + (q.w >> 16);
        const FvPair<W> sa0 = load_fv(fv + a0), sb0 = load_fv(fv + b0);
        const FvPair<W> sa1 = load_fv(fv + a1), sb1 = load_fv(fv + b1);
        const FvPair<W> sa2 = load_fv(fv + a2), sb2 = load_fv(fv + b2);
        const FvPair<W> sa3 = load_fv(fv + a3), sb3 = load_fv(fv + b3);
        act(a0, b0, sa0, sb0);
        act(a1, b1, sa1, sb1);
        act(a2, b2, sa2, sb2);
        act(a3, b3, sa3, sb3);
    }
}

// ms_sweep_unit over the unit's live chunks only: chunk c (its 16-byte
// groups 64c..64c+63; chunk 0 also the unaligned head and tail records) is
// skipped when bit c of dead[ui] is set -- every record in it had both ends
// visited by every query (qmask) at an earlier level, so it can discover
// nothing again.  With `mark`, the chunks found so in this sweep are marked
// for the levels after it (dead is written by other warps meanwhile: read
// through L2).
template <class W>
__device__ __forceinline__ void ms_sweep_unit_live(const gs_unit d, uint32_t ui, const uint32_t* __restrict__ base,
                                                   FvPair<W>* fv, W* next, int directed, uint32_t lane,
                                                   uint8_t* dead, bool mark, W qmask) {
    const uint32_t rb = (d.rc >> 16) << 16, cb = (d.rc & 0xFFFFu) << 16;
    uint32_t allv = 1;   // every record this lane visited has both ends visited by every query
    auto act = [&](uint32_t a, uint32_t b, const FvPair<W>& sa, const FvPair<W>& sb) {
        const W nb = sa.f & ~sb.vis;
        if (nb) atomicOr(next + b, nb);
        if (!directed) {            // the half grid stores each edge once
            const W na = sb.f & ~sa.vis;
            if (na) atomicOr(next + a, na);
        }
        allv &= (W)(sa.vis & sb.vis) == qmask ? 1u : 0u;
    };
    auto one = [&](uint32_t r) {
        const uint32_t a = rb + (r & 0xFFFFu), b = cb + (r >> 16);
        act(a, b, load_fv(fv + a), load_fv(fv + b));
    };
    const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
    uint64_t ab = (b + 3) & ~3ull;
    if (ab > e) ab = e;
    uint64_t ae = e & ~3ull;
    if (ae < ab) ae = ab;
    const uint4* r4 = reinterpret_cast<const uint4*>(base + ab);
    const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
    const uint32_t dd = __ldcg(dead + ui);
    const uint32_t nch = n4 ? (n4 + 63) >> 6 : 1;   // <= 8: a unit holds <= kUnitRecords records
    uint32_t todo = ((1u << nch) - 1u) & ~dd;
    if (!(dd & 1u)) {
        if (b + lane < ab) one(__ldcs(base + b + lane));
        if (ae + lane < e) one(__ldcs(base + ae + lane));
    }
    uint32_t newdead = 0;
    while (todo) {   // warp-uniform
        const uint32_t c = __ffs(todo) - 1;
        todo &= todo - 1;
        const uint32_t kend = min(n4, (c + 1) << 6);
        for (uint32_t k = (c << 6) + lane; k < kend; k += 32) {
            const uint4 q = load_stream(r4 + k);
            const uint32_t a0 = rb + (q.x & 0xFFFFu), b0 = cb + (q.x >> 16);
            const uint32_t a1 = rb + (q.y & 0xFFFFu), b1 = cb + (q.y >> 16);
            const uint32_t a2 = rb + (q.z & 0xFFFFu), b2 = cb + (q.z >> 16);
            const uint32_t a3 = rb + (q.w & 0xFFFFu), b3 = cb + (q.w >> 16);
            const FvPair<W> sa0 = load_fv(fv + a0), sb0 = load_fv(fv + b0);
            const FvPair<W> sa1 = load_fv(fv + a1), sb1 = load_fv(fv + b1);
            const FvPair<W> sa2 = load_fv(fv + a2), sb2 = load_fv(fv + b2);
            const FvPair<W> sa3 = load_fv(fv + a3), sb3 = load_fv(fv + b3);
            act(a0, b0, sa0, sb0);
            act(a1, b1, sa1, sb1);
            act(a2, b2, sa2, sb2);
            act(a3, b3, sa3, sb3);
        }
        if (mark) {
            if (__all_sync(kFull, allv)) newdead |= 1u << c;
            allv = 1;
        }
    }
    if (mark && lane == 0 && newdead)
        atomicOr(reinterpret_cast<unsigned int*>(dead) + (ui >> 2), newdead << ((ui & 3u) << 3));
}

// KcoreOp for a persistent kernel: the removed bits and window flags change
// between phases, so they are read through L2 (never the non-coherent path).
struct KcoreOpL2 {
    int32_t* deg;
    const uint32_t* removed;
    const uint8_t* act;
    struct Item {
        uint32_t rb, cb;
        bool fr, fc;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.fr = __ldcg(act + row) != 0;     // gstore.cpp:2773-2782
        c.fc = __ldcg(act + col) != 0;
        c.rb = row << 16;
        c.cb = col << 16;
        return c.fr || c.fc;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (c.fr && (__ldcg(removed + (a >> 5)) >> (a & 31) & 1u)) atomicSub(deg + b, 1);  // kcore.cpp:77-78
        if (c.fc && (__ldcg(removed + (b >> 5)) >> (b & 31) & 1u)) atomicSub(deg + a, 1);  // kcore.cpp:90-91
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

}  // namespace gsops
