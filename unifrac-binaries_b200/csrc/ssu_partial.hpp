// Partial results on disk: the reference's version-2 partial file
// (src/api.hpp:22-23, 816-857; src/api.cpp:1972-2428), LZ4 blocks through
// ssu_lz4.  Layout, all integers little-endian uint32:
//   header   magic 0x088ABA02, n_samples, n_stripes, stripe_start,
//            stripe_total, is_upper_triangle, id bytes, compressed id bytes
//   ids      one LZ4 block of the sample ids, each with its terminating NUL
//   stripes  per stripe: compressed size, then one LZ4 block of n_samples
//            doubles
//   footer   magic
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "unifrac_b200.h"

namespace ssu {

// Byte offset of every stripe's size field in a partial file, starting from
// the first stripe's (partial_dyn_mat_t::offsets[0]); read_error when the
// file ends early.
IOStatus partial_stripe_offsets(const char *filename, uint64_t first, uint32_t n_stripes,
                                std::vector<uint64_t> &offsets);

// One stripe (n_samples doubles) whose size field starts at `offset`.
IOStatus partial_read_stripe_at(const char *filename, uint64_t offset, uint32_t n_samples, double *out);

// The reference's check_partial (src/api.cpp:2322-2394): same sample count,
// stripe total, triangle flag and ids in every partial, no stripe twice,
// every stripe present.
MergeStatus partial_check(const partial_dyn_mat_t *const *mats, int n, bool verbose);

}  // namespace ssu
