"""Branch lengths as two products of bytes (ssu_digits.hpp), the arithmetic
under the tensor-core unweighted contraction: every chunk-scaled length
q < 2^23 must come back as q = 256 u v + s t with u, v, s, t in [0, 255]
and u v, s t <= 32,767 (so a chunk of at most 512 blocks x 128 nodes keeps
its int32 product sums exact).  A host program built from the header checks
every q on the CPU; a wrong digit would be a wrong distance, not a fault."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "unifrac-binaries_b200", "csrc")

PROBE = r"""
#include <cstdio>
#include "ssu_digits.hpp"
int main() {
    using namespace ssu::digits;
    uint8_t d[4];
    for (uint32_t q = 0; q < (1u << kBits); q++) {
        if (!split_length(q, d)) { std::printf("no form %u\n", q); return 1; }
        const uint32_t uv = uint32_t(d[0]) * d[2], st = uint32_t(d[1]) * d[3];
        if (256u * uv + st != q || uv > kMaxPart || st > kMaxPart) { std::printf("bad %u\n", q); return 2; }
    }
    if (split_length(1u << kBits, d)) { std::printf("accepted 2^23\n"); return 3; }
    static_assert(512ll * 128 * kMaxPart < (1ll << 31), "chunk sums must stay exact in int32");
    std::printf("ok\n");
    return 0;
}
"""


def test_every_length_below_2_23_has_a_byte_product_form(tmp_path):
    src = tmp_path / "digits.cpp"
    src.write_text(PROBE)
    exe = tmp_path / "digits"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
