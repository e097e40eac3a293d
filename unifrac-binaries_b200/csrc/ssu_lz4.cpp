// LZ4 block codec written from the LZ4 block format specification.
//
// A block is a series of sequences.  Each sequence: a token byte (high 4
// bits literal count, low 4 bits match length - 4; 15 means more length
// bytes follow, each added, a byte below 255 ending the run), the literals,
// then a 2-byte little-endian match offset (1..65535 back into the output)
// and the extra match-length bytes.  The last sequence holds literals only.
// End-of-block rules: the last 5 bytes are always literals and the last match
// starts at least 12 bytes before the end of the input.
#include "ssu_lz4.hpp"

#include <cstring>
#include <vector>

namespace ssu {
namespace {

constexpr size_t kMinMatch = 4;
constexpr size_t kLastLiterals = 5;
constexpr size_t kMatchSafety = 12;  // no match may start in the last 12 bytes
constexpr int kHashBits = 16;

inline uint32_t read32(const uint8_t *p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
inline uint32_t hash4(uint32_t v) { return (v * 2654435761u) >> (32 - kHashBits); }

// Length field continuation: `len` beyond the token's 15, as 255-bytes + rest.
inline uint8_t *put_length(uint8_t *op, size_t len) {
    while (len >= 255) {
        *op++ = 255;
        len -= 255;
    }
    *op++ = static_cast<uint8_t>(len);
    return op;
}

}  // namespace

size_t lz4_bound(size_t n) { return n + n / 255 + 16; }

size_t lz4_compress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    if (cap < lz4_bound(n)) return 0;
    uint8_t *op = dst;
    size_t anchor = 0;  // first literal not yet emitted
    if (n >= kMatchSafety + 1) {
        std::vector<int64_t> table(size_t(1) << kHashBits, -1);
        const size_t match_limit = n - kMatchSafety;  // last position a match may start at
        size_t ip = 0;
        while (ip < match_limit) {
            const uint32_t seq = read32(src + ip);
            const uint32_t h = hash4(seq);
            const int64_t cand = table[h];
            table[h] = static_cast<int64_t>(ip);
            if (cand < 0 || ip - static_cast<size_t>(cand) > 65535 || read32(src + cand) != seq) {
                ip++;
                continue;
            }
            // extend the match forward, stopping before the last literals
            size_t len = kMinMatch;
            const size_t max_len = n - kLastLiterals - ip;
            while (len < max_len && src[cand + len] == src[ip + len]) len++;
            // sequence: literals [anchor, ip), match (ip - cand, len)
            const size_t lit = ip - anchor;
            uint8_t *token = op++;
            *token = static_cast<uint8_t>((lit >= 15 ? 15 : lit) << 4);
            if (lit >= 15) op = put_length(op, lit - 15);
            std::memcpy(op, src + anchor, lit);
            op += lit;
            const size_t off = ip - static_cast<size_t>(cand);
            *op++ = static_cast<uint8_t>(off & 0xFF);
            *op++ = static_cast<uint8_t>(off >> 8);
            const size_t ml = len - kMinMatch;
            *token |= static_cast<uint8_t>(ml >= 15 ? 15 : ml);
            if (ml >= 15) op = put_length(op, ml - 15);
            ip += len;
            anchor = ip;
            // seed the table inside the match so later repeats find it
            if (ip - 2 < match_limit) table[hash4(read32(src + ip - 2))] = static_cast<int64_t>(ip - 2);
        }
    }
    // the last sequence: literals only
    const size_t lit = n - anchor;
    *op++ = static_cast<uint8_t>((lit >= 15 ? 15 : lit) << 4);
    if (lit >= 15) op = put_length(op, lit - 15);
    std::memcpy(op, src + anchor, lit);
    op += lit;
    return static_cast<size_t>(op - dst);
}

long long lz4_decompress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    size_t ip = 0, op = 0;
    if (n == 0) return -1;
    while (ip < n) {
        const uint8_t token = src[ip++];
        size_t lit = token >> 4;
        if (lit == 15) {
            uint8_t b;
            do {
                if (ip >= n) return -1;
                b = src[ip++];
                lit += b;
            } while (b == 255);
        }
        if (lit > n - ip || lit > cap - op) return -1;
        std::memcpy(dst + op, src + ip, lit);
        ip += lit;
        op += lit;
        if (ip == n) break;  // the last sequence has no match
        if (n - ip < 2) return -1;
        const size_t off = static_cast<size_t>(src[ip]) | (static_cast<size_t>(src[ip + 1]) << 8);
        ip += 2;
        if (off == 0 || off > op) return -1;
        size_t ml = (token & 0x0F);
        if (ml == 15) {
            uint8_t b;
            do {
                if (ip >= n) return -1;
                b = src[ip++];
                ml += b;
            } while (b == 255);
        }
        ml += kMinMatch;
        if (ml > cap - op) return -1;
        // byte by byte: the match may overlap the bytes it produces
        const size_t from = op - off;
        for (size_t i = 0; i < ml; i++) dst[op + i] = dst[from + i];
        op += ml;
    }
    return static_cast<long long>(op);
}

}  // namespace ssu
