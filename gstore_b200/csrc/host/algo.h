// The reference's per-algorithm plug-in interface (algo.h:38-44), kept for
// drop-in use, with each algorithm's state living in HBM behind the C ABI of
// libgstore_cuda.so.
//
//   reference                         here
//   algo_t::algo_mem_part(segment*)   enqueue the device sweep of the segment's
//                                     tile runs (nullptr / empty = all resident)
//   iteration_finalize()              device finalize + one 8-byte read
//   calc_part_needed()                tile activity is tracked on the device
//   vertex_active(v)                  answered from the device state
//
// Threading: the reference enters algo_mem_part from every OpenMP thread;
// here one host thread calls it once per segment and the GPU does the split.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gstore_cuda.h"

typedef uint64_t index_t;
typedef uint64_t vertex_t;
typedef uint64_t part_id;

// part_meta_t (gstore.h:563-568): a run of consecutive tiles in file order.
class part_meta_t {
public:
    size_t offset;
    part_id start;
    part_id end;
};

// segment (gstore.h:578-583): the runs held in one staging buffer.
class segment {
public:
    char* buf;
    index_t ctx_count;
    part_meta_t* meta;
};

// Throws nothing: failures are recorded and reported by status().
class algo_t {
public:
    virtual ~algo_t();
    virtual void algo_mem_part(segment* seg) = 0;
    virtual int iteration_finalize() = 0;
    void calc_part_needed() {}
    virtual bool vertex_active(vertex_t v);
    gs_status status() const { return status_; }
    const std::string& error() const { return error_; }
    gs_state* state() const { return st_; }

protected:
    bool check(gs_status s);
    void sweep(segment* seg);
    gs_ctx* ctx_ = nullptr;
    gs_state* st_ = nullptr;
    gs_status status_ = GS_OK;
    std::string error_;
};

// bfs_t (bfs.h:40-56): depth_t levels, root = 1, INFTY = 0.
class bfs_t : public algo_t {
public:
    void init(gs_ctx* ctx, gs_graph* g, vertex_t root);
    void algo_mem_part(segment* seg) override;
    int iteration_finalize() override;   // 1 when the frontier is empty
    uint8_t level = 1;
    int64_t front_count = 0;
};

// pr_t (pr.h:40-52): not an algo_t in the reference either.
class pr_t {
public:
    void init(gs_ctx* ctx, gs_graph* g, int iteration_count, bool compat);
    void algo_mem_part(segment* seg);
    void iteration_finalize(int current_iteration);
    gs_status status() const { return status_; }
    const std::string& error() const { return error_; }
    gs_state* state() const { return st_; }
    ~pr_t();

private:
    gs_ctx* ctx_ = nullptr;
    gs_state* st_ = nullptr;
    gs_status status_ = GS_OK;
    std::string error_;
};

// kcore_t (kcore.h:37-53).
class kcore_t : public algo_t {
public:
    void init(gs_ctx* ctx, gs_graph* g, int kc);
    void algo_mem_part(segment* seg) override;
    int iteration_finalize() override;   // vertices removed this round
    int kc = 10;
};

// wcc2_t (wcc.h:71-102).
class wcc2_t : public algo_t {
public:
    void init(gs_ctx* ctx, gs_graph* g);
    void algo_mem_part(segment* seg) override;
    int iteration_finalize() override;   // 0 once no label changed
    uint64_t wcc_count = 0;
};

// bfs2_t (bfs2.h:38-52): label-correcting BFS ("-j 30").
class bfs2_t : public algo_t {
public:
    void init(gs_ctx* ctx, gs_graph* g, vertex_t root);
    void algo_mem_part(segment* seg) override;
    int iteration_finalize() override;   // changes in the sweep; 0 ends the run
    uint8_t level = 1;
};

// traverse_t (traverse.h:38-50): single-colour propagation ("-j 4").
class traverse_t : public algo_t {
public:
    void init(gs_ctx* ctx, gs_graph* g, vertex_t pivot);
    void algo_mem_part(segment* seg) override;
    int iteration_finalize() override;   // vertices coloured in the sweep; 0 ends the run
    int iteration = 0;
};
