// BIOM 2.x tables stored in HDF5 files, read without the HDF5 library.
//
// The reference opens a table file with the HDF5 C++ API (src/biom.cpp:18-255)
// and reads five datasets: /observation/ids and /sample/ids (variable-length
// strings), and the observation-major CSR /observation/matrix/indptr,
// /observation/matrix/indices and /observation/matrix/data.  This reader
// parses the subset of the HDF5 file format those files use: superblock
// versions 0 and 1, version-1 object headers with continuation blocks, groups
// held as symbol tables (version-1 B-trees, symbol-table nodes, local heaps),
// contiguous, compact and chunked (version-1 B-tree index) dataset layouts
// (layout message versions 1-3), the deflate, shuffle and Fletcher-32
// filters, little-endian integer and floating-point element types, and
// fixed- or variable-length strings (the latter through global heap
// collections).  Other files are refused with a message, never guessed at.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ssu_table.hpp"

namespace ssu {

// Fills `out` (an owning table, totals computed) from a BIOM 2.x HDF5 file.
// Returns false and sets `err` when the file cannot be read as one.
bool read_biom_hdf5(const std::string &path, Table &out, std::string &err);

// One dataset of such a file, e.g. the reference's own output files
// (src/api.cpp:1160-1290: "matrix", "order", "pcoa_eigvals", "pcoa_samples",
// "pcoa_proportion_explained", "stat_*").  Compact and contiguous layouts of
// any rank, chunked ones of rank 1.  Numbers come back as doubles in storage
// (row-major) order, strings as strings.
struct H5Data {
    std::vector<uint64_t> dims;
    bool is_string = false;
    std::vector<double> values;
    std::vector<std::string> strings;
};
bool read_hdf5_dataset(const std::string &path, const std::string &name, H5Data &out, std::string &err);

}  // namespace ssu
