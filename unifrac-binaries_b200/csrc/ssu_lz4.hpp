// LZ4 block format (the published LZ4 block specification), as the partial
// result files use it (src/api.cpp:1972-2245 calls LZ4_compress_default and
// LZ4_decompress_safe on each block).  Any conforming LZ4 block decoder reads
// what lz4_compress writes, and lz4_decompress reads any conforming block.
#pragma once

#include <cstddef>
#include <cstdint>

namespace ssu {

// Worst-case compressed size of n input bytes.
size_t lz4_bound(size_t n);

// Compresses src[0, n) into dst (capacity cap >= lz4_bound(n)); returns the
// compressed size, 0 on failure.
size_t lz4_compress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap);

// Decompresses a block of `n` bytes into dst (capacity cap); returns the
// decompressed size, or -1 for a malformed block or one that does not fit.
long long lz4_decompress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap);

}  // namespace ssu
