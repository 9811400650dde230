#include "algo.h"

#include <algorithm>
#include <iostream>

algo_t::~algo_t() {
    if (st_) gs_state_free(st_);
}

bool algo_t::vertex_active(vertex_t) { return false; }

bool algo_t::check(gs_status s) {
    if (s != GS_OK && status_ == GS_OK) {
        status_ = s;
        error_ = gs_last_error(ctx_);
    }
    return s == GS_OK;
}

void algo_t::sweep(segment* seg) {
    if (status_ != GS_OK) return;
    if (seg && seg->ctx_count) {
        std::vector<gs_segment> runs(seg->ctx_count);
        for (index_t k = 0; k < seg->ctx_count; ++k) {
            runs[k].part_start = seg->meta[k].start;
            runs[k].part_end = seg->meta[k].end;
        }
        check(gs_sweep(st_, runs.data(), (int)runs.size()));
    } else {
        check(gs_sweep(st_, nullptr, 0));
    }
}

// ------------------------------------------------------------------ BFS ---
void bfs_t::init(gs_ctx* ctx, gs_graph* g, vertex_t root) {
    ctx_ = ctx;
    check(gs_state_create(g, GS_ALGO_BFS, (int64_t)root, &st_));
    level = 1;
    std::cout << "Root = " << root << std::endl;   // bfs.cpp:175
}

void bfs_t::algo_mem_part(segment* seg) { sweep(seg); }

int bfs_t::iteration_finalize() {
    if (status_ != GS_OK) return 1;
    int done = 0;
    if (!check(gs_finalize(st_, &front_count, &done))) return 1;
    // bfs.cpp:296-297
    std::cout << "level: " << (int)level << " frontier count: " << front_count << std::endl;
    if (done) return 1;
    ++level;
    return 0;
}

// ------------------------------------------------------------- PageRank ---
void pr_t::init(gs_ctx* ctx, gs_graph* g, int iteration_count, bool compat) {
    ctx_ = ctx;
    status_ = gs_state_create(g, GS_ALGO_PAGERANK, iteration_count, &st_);
    if (status_ == GS_OK && compat) status_ = gs_pagerank_compat(st_, 1);
    if (status_ != GS_OK) error_ = gs_last_error(ctx);
}

pr_t::~pr_t() {
    if (st_) gs_state_free(st_);
}

void pr_t::algo_mem_part(segment* seg) {
    if (status_ != GS_OK) return;
    (void)seg;
    status_ = gs_sweep(st_, nullptr, 0);
    if (status_ != GS_OK) error_ = gs_last_error(ctx_);
}

void pr_t::iteration_finalize(int) {
    if (status_ != GS_OK) return;
    int64_t f;
    int d;
    status_ = gs_finalize(st_, &f, &d);
    if (status_ != GS_OK) error_ = gs_last_error(ctx_);
}

// --------------------------------------------------------------- k-core ---
void kcore_t::init(gs_ctx* ctx, gs_graph* g, int k) {
    ctx_ = ctx;
    kc = k;
    check(gs_state_create(g, GS_ALGO_KCORE, k, &st_));
}

void kcore_t::algo_mem_part(segment* seg) { sweep(seg); }

int kcore_t::iteration_finalize() {
    if (status_ != GS_OK) return 0;
    int64_t removed = 0;
    int done = 0;
    if (!check(gs_finalize(st_, &removed, &done))) return 0;
    std::cout << " frontier count: " << removed << std::endl;   // kcore.cpp:212
    return (int)removed;
}

// ------------------------------------------------------------------ WCC ---
void wcc2_t::init(gs_ctx* ctx, gs_graph* g) {
    ctx_ = ctx;
    check(gs_state_create(g, GS_ALGO_WCC, 0, &st_));
}

void wcc2_t::algo_mem_part(segment* seg) { sweep(seg); }

int wcc2_t::iteration_finalize() {
    if (status_ != GS_OK) return 0;
    int64_t changed = 0;
    int done = 0;
    if (!check(gs_finalize(st_, &changed, &done))) return 0;
    std::cout << "level: " << " frontier count: " << changed << std::endl << std::endl;  // wcc.cpp:290-292
    if (done) {
        if (!check(gs_result_count(st_, &wcc_count))) return 0;
        std::cout << "WCC count = " << wcc_count << std::endl;   // wcc.cpp:336
        return 0;
    }
    return 1;
}

// ----------------------------------------------------------------- bfs2 ---
void bfs2_t::init(gs_ctx* ctx, gs_graph* g, vertex_t root) {
    ctx_ = ctx;
    check(gs_state_create(g, GS_ALGO_BFS2, (int64_t)root, &st_));
    level = 1;
    std::cout << "Root = " << root << std::endl;   // bfs2.cpp:75
}

void bfs2_t::algo_mem_part(segment* seg) { sweep(seg); }

int bfs2_t::iteration_finalize() {
    if (status_ != GS_OK) return 0;
    int64_t changed = 0;
    int done = 0;
    if (!check(gs_finalize(st_, &changed, &done))) return 0;
    std::cout << "level: " << (int)level << " frontier count: " << changed << std::endl;   // bfs2.cpp:140-141
    if (done) return 0;
    ++level;
    return (int)std::min<int64_t>(changed, 1 << 30);
}

// ------------------------------------------------------------- traverse ---
void traverse_t::init(gs_ctx* ctx, gs_graph* g, vertex_t pivot) {
    ctx_ = ctx;
    check(gs_state_create(g, GS_ALGO_TRAVERSE, (int64_t)pivot, &st_));
    iteration = 0;
}

void traverse_t::algo_mem_part(segment* seg) { sweep(seg); }

int traverse_t::iteration_finalize() {
    if (status_ != GS_OK) return 0;
    int64_t colored = 0;
    int done = 0;
    if (!check(gs_finalize(st_, &colored, &done))) return 0;
    // traverse.cpp:199-201
    std::cout << "level: " << iteration << " frontier count: " << colored << std::endl << std::endl;
    if (done) return 0;
    ++iteration;
    return (int)std::min<int64_t>(colored, 1 << 30);
}
