#include "tilefile.h"

#include <cstdio>
#include <sys/stat.h>

namespace {

std::string file_size(const std::string& path, uint64_t* bytes) {
    struct stat st;
    if (stat(path.c_str(), &st) != 0) return "cannot stat " + path;
    *bytes = (uint64_t)st.st_size;
    return "";
}

template <class T>
std::string read_all(const std::string& path, uint64_t count, std::vector<T>* out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    out->resize(count);
    uint64_t got = count ? std::fread(out->data(), sizeof(T), count, f) : 0;
    std::fclose(f);
    if (got != count) return "short read on " + path;
    return "";
}

template <class T>
std::string write_all(const std::string& path, const T* data, uint64_t count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot create " + path;
    uint64_t put = count ? std::fwrite(data, sizeof(T), count, f) : 0;
    std::fclose(f);
    if (put != count) return "short write on " + path;
    return "";
}

}  // namespace

std::string tile_file_size(const std::string& path, uint64_t* bytes) { return file_size(path, bytes); }

std::string read_tile_files(const std::string& prefix, uint64_t expected_start_entries, uint64_t vert_count,
                            bool want_degree, tile_files* out, bool want_grid) {
    uint64_t sb = 0, gb = 0;
    std::string err = file_size(prefix + ".start", &sb);
    if (!err.empty()) return err;
    if (sb % 8) return prefix + ".start size is not a multiple of 8";
    if (sb / 8 != expected_start_entries)
        return prefix + ".start has " + std::to_string(sb / 8) + " entries; the tile geometry needs " +
               std::to_string(expected_start_entries) + " (check -s/-v)";
    err = file_size(prefix + ".grid", &gb);
    if (!err.empty()) return err;
    if (gb % 4) return prefix + ".grid size is not a multiple of 4";
    err = read_all(prefix + ".start", sb / 8, &out->start);
    if (!err.empty()) return err;
    if (out->start.back() != gb / 4)
        return "last .start entry (" + std::to_string(out->start.back()) + ") != records in .grid (" +
               std::to_string(gb / 4) + ")";
    out->grid.clear();
    if (want_grid) {
        err = read_all(prefix + ".grid", gb / 4, &out->grid);
        if (!err.empty()) return err;
    }
    out->degree.clear();
    if (want_degree) {
        uint64_t db = 0;
        err = file_size(prefix + ".degree", &db);
        if (!err.empty()) return err;
        // read_degree_in_mem reads vert_count entries (gstore.cpp:2999-3010);
        // a shorter file leaves the tail at zero as calloc does there.
        uint64_t n = db / 4 < vert_count ? db / 4 : vert_count;
        err = read_all(prefix + ".degree", n, &out->degree);
        if (!err.empty()) return err;
        out->degree.resize(vert_count, 0);
    }
    return "";
}

std::string write_tile_files(const std::string& prefix, const tile_files& tf) {
    std::string err = write_all(prefix + ".grid", tf.grid.data(), tf.grid.size());
    if (!err.empty()) return err;
    err = write_all(prefix + ".start", tf.start.data(), tf.start.size());
    if (!err.empty()) return err;
    err = write_all(prefix + ".degree", tf.degree.data(), tf.degree.size());
    if (!err.empty()) return err;
    // compress_degree (gstore.cpp:1461-1489): int16 degrees, with every degree
    // above 32767 moved to .bdegree and referenced as -index; entry 0 of
    // .bdegree is a placeholder (6000).
    std::vector<int16_t> sdeg(tf.degree.size());
    std::vector<int32_t> bdeg(1, 6000);
    for (size_t v = 0; v < tf.degree.size(); ++v) {
        if (tf.degree[v] > 32767) {
            sdeg[v] = (int16_t)(-(int32_t)bdeg.size());
            bdeg.push_back(tf.degree[v]);
        } else {
            sdeg[v] = (int16_t)tf.degree[v];
        }
    }
    err = write_all(prefix + ".sdegree", sdeg.data(), sdeg.size());
    if (!err.empty()) return err;
    return write_all(prefix + ".bdegree", bdeg.data(), bdeg.size());
}

std::string read_edge_list(const std::string& path, std::vector<uint32_t>* pairs) {
    uint64_t b = 0;
    std::string err = file_size(path, &b);
    if (!err.empty()) return err;
    if (b % 8) return path + " size is not a multiple of 8 (gedge_t)";
    return read_all(path, b / 4, pairs);
}
