// Tile-file loader/saver for the reference's on-disk format.
//   <prefix>.start  uint64 x (tiles + 1)   grid::save_start_files (gstore.cpp:2899-2908)
//   <prefix>.grid   uint32 x records       grid::save_grid        (gstore.cpp:2818-2829)
//   <prefix>.degree int32  x V             grid::save_degree_files (gstore.cpp:2911-2917)
//   <prefix>.sdegree/.bdegree              compress_degree         (gstore.cpp:1461-1489)
#pragma once
#include <cstdint>
#include <string>
#include <vector>

struct tile_files {
    std::vector<uint64_t> start;
    std::vector<uint32_t> grid;
    std::vector<int32_t> degree;   // empty when not loaded
};

// Returns "" on success, otherwise the reason (missing file, size not a
// multiple of the element, entry count not matching the geometry).  With
// want_grid false the .grid file is checked but not read (out->grid stays
// empty): the records then stream from the file.
std::string read_tile_files(const std::string& prefix, uint64_t expected_start_entries,
                            uint64_t vert_count, bool want_degree, tile_files* out, bool want_grid = true);

// Size of a file in bytes ("" on success).
std::string tile_file_size(const std::string& path, uint64_t* bytes);

// Writes .grid/.start/.degree and the compressed .sdegree/.bdegree pair.
std::string write_tile_files(const std::string& prefix, const tile_files& tf);

// Reads a binary edge list of gedge_t {uint32 v0, v1} (gstore.h:255-279).
std::string read_edge_list(const std::string& path, std::vector<uint32_t>* pairs);
