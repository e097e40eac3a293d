// Branch lengths as two products of bytes, for the tensor-core unweighted
// contraction: a length scaled to a chunk's fixed point, q < 2^23, is
// written q = 256 u v + s t with u, v, s, t in [0, 255], so two 8-bit
// products (u on one operand and v on the other, then s and t) carry 23
// bits where one would carry 16.  Plain C++ (no CUDA), so the host tests
// can check it over every q.
#pragma once

#include <algorithm>
#include <cstdint>
#include <iterator>

namespace ssu {
namespace digits {

constexpr int kBits = 23;             // fixed-point bits of a chunk's largest length
constexpr uint32_t kMaxPart = 32767;  // largest u v and s t (their sums over a chunk stay below 2^31)

// q (< 2^23) as 256 u v + s t with u v, s t <= 32767: d = {u, s, v, t}.
// p = u v runs down from q / 256 (s t = q - 256 p up from q mod 256) until
// both are products of two bytes; every q < 2^23 has such a pair within 112
// steps.  False if none is found (q out of range).
inline bool split_length(uint32_t q, uint8_t d[4]) {
    struct Factors {
        uint16_t f[kMaxPart + 1];  // u | v << 8 for p = u v, or 0xFFFF
        Factors() {
            std::fill(std::begin(f), std::end(f), static_cast<uint16_t>(0xFFFF));
            f[0] = 0;
            for (uint32_t u = 1; u < 256; u++)
                for (uint32_t v = u; v < 256 && u * v <= kMaxPart; v++)
                    if (f[u * v] == 0xFFFF) f[u * v] = static_cast<uint16_t>(u | (v << 8));
        }
    };
    static const Factors tab;
    if (q >= (1u << kBits)) return false;
    for (int64_t p = q >> 8, rest = q & 255; p >= 0 && rest <= static_cast<int64_t>(kMaxPart); p--, rest += 256) {
        if (p > static_cast<int64_t>(kMaxPart)) continue;
        const uint16_t a = tab.f[p], b = tab.f[rest];
        if (a == 0xFFFF || b == 0xFFFF) continue;
        d[0] = static_cast<uint8_t>(a & 0xFF);
        d[2] = static_cast<uint8_t>(a >> 8);
        d[1] = static_cast<uint8_t>(b & 0xFF);
        d[3] = static_cast<uint8_t>(b >> 8);
        return true;
    }
    return false;
}

}  // namespace digits
}  // namespace ssu
