// CUDA kernels of the B200 UniFrac engine (sm_100a).
//
// Data layout in HBM (one group of tables sharing the tree):
//   U[row][j]   proportion embedding, rows = non-root nodes (embedded rows
//               first, in postorder), j = column.  Table t of the group owns
//               columns [base_t, base_t + n_t); every base and every table's
//               width are multiples of 128, so each tile load is in bounds and
//               16-byte aligned; padding columns are zero.  `ld` = the group's
//               column count.
//   C[row][j]   raw-count embedding (variance-adjusted methods only).
//   P[w][j]     presence bits of 64 consecutive embedded rows (unweighted).
//   LUT[w][b][v] sum of the lengths selected by the bits of byte value v in
//               byte b of word w (unweighted), as the reference's 8-bit length
//               tables (src/unifrac_task_impl.hpp:1448-1514).
//
// The pair kernels compute d(k, l) for a square tile of sample pairs with the
// accumulators in registers across every embedded node, so the per-batch
// read-modify-write of the reference's stripe buffers
// (src/unifrac_task_impl.hpp:333-433) never reaches memory.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace ssu {
namespace dev {

// ------------------------------------------------------------- utilities

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- mbarriers
// Every wait on an mbarrier is bounded (clock64 budget): the caller records
// an error and stops instead of spinning for ever.

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 2-D tiled TMA load of the box at (x = column, y = row) into shared memory,
// completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}
// Bounded wait for the phase of `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long budget) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > budget) return false;
    return true;
}

// --------------------------------------------------------------- embedding

// One table of a group: where its CSR entries, its embedding columns and
// its result live.
struct TableDesc {
    uint64_t out_off;     // first element of the table's result in the output buffer
    uint64_t nnz_off;     // first CSR entry of the table in the concatenated indices/data
    uint32_t indptr_off;  // first indptr entry of the table
    uint32_t base;        // first embedding column of the table in its group
    uint32_t n;           // samples
    uint32_t pad;
};

// Tip rows: zero the row, then scatter the CSR entries of the tip's
// observation from every table of the group; proportions are data / total in
// fp64 and then rounded to T (src/biom_inmem.cpp:473-497).
// tip_obs[t * n_tables + i] = row of tip t's observation in table i, or -1.
// Presence masks written by the embedding (the sparse pair kernels' input):
// bit i of masks[w * E + row] is U[row][64 w + i] > 0, counts[row] the row's
// set bits; both zeroed before the embedding.  masks == nullptr: none.
struct MaskOut {
    unsigned long long *masks;
    uint32_t *counts;
    uint32_t E;
};

// bit i of x -> bit 2i, and bit i of the low 16 bits -> bit 4i
__device__ __forceinline__ unsigned long long spread2(uint32_t v) {
    unsigned long long x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
__device__ __forceinline__ unsigned long long spread4(uint32_t v) {
    unsigned long long x = v & 0xFFFFu;
    x = (x | (x << 24)) & 0x000000FF000000FFull;
    x = (x | (x << 12)) & 0x000F000F000F000Full;
    x = (x | (x << 6)) & 0x0303030303030303ull;
    x = (x | (x << 3)) & 0x1111111111111111ull;
    return x;
}

template <typename T, bool COUNTS>
__global__ void embed_tips_kernel(const uint32_t *__restrict__ tip_rows, const int32_t *__restrict__ tip_obs,
                                  uint32_t n_tips, uint32_t n_tables, const TableDesc *__restrict__ tables,
                                  const uint32_t *__restrict__ indptr, const uint32_t *__restrict__ indices,
                                  const double *__restrict__ data, const double *__restrict__ totals, bool normalize,
                                  T *__restrict__ U, T *__restrict__ C, uint64_t ld, MaskOut mo) {
    for (uint32_t t = blockIdx.x; t < n_tips; t += gridDim.x) {
        const uint64_t row = tip_rows[t];
        T *u = U + row * ld;
        T *c = COUNTS ? C + row * ld : nullptr;
        for (uint64_t j = threadIdx.x; j < ld; j += blockDim.x) {
            u[j] = T(0);
            if (COUNTS) c[j] = T(0);
        }
        __syncthreads();
        for (uint32_t i = 0; i < n_tables; i++) {
            const int32_t r = tip_obs[static_cast<uint64_t>(t) * n_tables + i];
            if (r < 0) continue;
            const TableDesc td = tables[i];
            const uint32_t *ip = indptr + td.indptr_off;
            for (uint32_t q = ip[r] + threadIdx.x; q < ip[r + 1]; q += blockDim.x) {
                const uint64_t qa = td.nnz_off + q;
                const uint32_t j = td.base + indices[qa];
                const double v = data[qa];
                const T uv = normalize ? static_cast<T>(v / totals[j]) : static_cast<T>(v);
                u[j] = uv;
                if (COUNTS) c[j] = static_cast<T>(v);
                if (mo.masks && row < mo.E && uv > T(0)) {
                    atomicOr(mo.masks + (j >> 6) * mo.E + row, 1ull << (j & 63));
                    atomicAdd(mo.counts + row, 1u);
                }
            }
        }
        __syncthreads();
    }
}

template <typename T> struct Vec16;
template <> struct Vec16<double> {
    using type = double2;
    static constexpr int n = 2;
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
};
template <> struct Vec16<float> {
    using type = float4;
    static constexpr int n = 4;
    __device__ static float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ static float4 add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
};

// One tree level: every internal row is the sum of its children, left child
// first onto zero (src/unifrac_internal.cpp:240-257), 16 bytes per thread.
template <typename T, bool COUNTS>
__global__ void embed_level_kernel(const uint32_t *__restrict__ rows, uint32_t n_rows,
                                   const uint32_t *__restrict__ child_ptr, const uint32_t *__restrict__ child_rows,
                                   T *__restrict__ U, T *__restrict__ C, uint64_t ld, uint32_t col_blocks, MaskOut mo) {
    using V = typename Vec16<T>::type;
    const uint64_t nvec = ld / Vec16<T>::n;
    const uint64_t total = static_cast<uint64_t>(n_rows) * col_blocks;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t b = blockIdx.x; b < total; b += gridDim.x) {
        const uint32_t row = rows[b / col_blocks];
        const uint64_t v = (b % col_blocks) * blockDim.x + threadIdx.x;
        const bool ok = v < nvec;
        V s = Vec16<T>::zero();
        V sc = Vec16<T>::zero();
        if (ok) {
            for (uint32_t c = child_ptr[row]; c < child_ptr[row + 1]; c++) {
                const uint64_t cr = child_rows[c];
                s = Vec16<T>::add(s, reinterpret_cast<const V *>(U + cr * ld)[v]);
                if (COUNTS) sc = Vec16<T>::add(sc, reinterpret_cast<const V *>(C + cr * ld)[v]);
            }
            reinterpret_cast<V *>(U + static_cast<uint64_t>(row) * ld)[v] = s;
            if (COUNTS) reinterpret_cast<V *>(C + static_cast<uint64_t>(row) * ld)[v] = sc;
        }
        if (mo.masks) {
            // the warp's 32 vectors are 64 (fp64) or 128 (fp32) consecutive
            // columns starting on a 64-column word
            const uint64_t w0 = (v - lane) * Vec16<T>::n / 64;
            if constexpr (sizeof(T) == 8) {
                const uint32_t bx = __ballot_sync(0xffffffffu, ok && s.x > T(0));
                const uint32_t by = __ballot_sync(0xffffffffu, ok && s.y > T(0));
                if (lane == 0 && row < mo.E) {
                    const unsigned long long word = spread2(bx) | (spread2(by) << 1);
                    if (word) {
                        mo.masks[w0 * mo.E + row] = word;
                        atomicAdd(mo.counts + row, static_cast<uint32_t>(__popcll(word)));
                    }
                }
            } else {
                const uint32_t b0 = __ballot_sync(0xffffffffu, ok && s.x > T(0));
                const uint32_t b1 = __ballot_sync(0xffffffffu, ok && s.y > T(0));
                const uint32_t b2 = __ballot_sync(0xffffffffu, ok && s.z > T(0));
                const uint32_t b3 = __ballot_sync(0xffffffffu, ok && s.w > T(0));
                if (lane < 2 && row < mo.E) {
                    const uint32_t sh = 16 * lane;
                    const unsigned long long word = spread4(b0 >> sh) | (spread4(b1 >> sh) << 1) |
                                                    (spread4(b2 >> sh) << 2) | (spread4(b3 >> sh) << 3);
                    if (word && (w0 + lane) * 64 < ld) {
                        mo.masks[(w0 + lane) * mo.E + row] = word;
                        atomicAdd(mo.counts + row, static_cast<uint32_t>(__popcll(word)));
                    }
                }
            }
        }
    }
}

// W[j] = sum_e L_e u_e[j] over embedded rows, in fixed row chunks (partial
// sums, then an in-order reduction), the one-sided sums of
// src/unifrac_task_impl.hpp:51-103.  With per-table lengths (block_table
// set, 128 threads per block) a block's columns all belong to the table
// block_table[blockIdx.x].
template <typename T>
__global__ void weighted_sums_partial_kernel(const T *__restrict__ U, const T *__restrict__ len, uint32_t E,
                                             uint64_t ld, uint32_t chunk, T *__restrict__ partial,
                                             const uint32_t *__restrict__ block_table, uint64_t len_stride) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    const T *L = block_table ? len + block_table[blockIdx.x] * len_stride : len;
    const uint32_t e0 = blockIdx.y * chunk;
    const uint32_t e1 = min(E, e0 + chunk);
    T s = T(0);
    for (uint32_t e = e0; e < e1; e++) s = fma(U[static_cast<uint64_t>(e) * ld + j], L[e], s);
    partial[static_cast<uint64_t>(blockIdx.y) * ld + j] = s;
}

template <typename T>
__global__ void reduce_partials_kernel(const T *__restrict__ partial, uint32_t n_parts, uint64_t ld,
                                       T *__restrict__ out) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    T s = T(0);
    for (uint32_t p = 0; p < n_parts; p++) s += partial[static_cast<uint64_t>(p) * ld + j];
    out[j] = s;
}

// Presence bits of 64 embedded rows per word: bit b of P[w][j] is u[64w+b][j] > 0.
template <typename T>
__global__ void pack_presence_kernel(const T *__restrict__ U, uint32_t E, uint64_t ld, uint32_t n_words,
                                     unsigned long long *__restrict__ P) {
    const uint64_t total = static_cast<uint64_t>(n_words) * ld;
    for (uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t w = idx / ld, j = idx % ld;
        unsigned long long bits = 0ull;
        const uint32_t e0 = static_cast<uint32_t>(w * 64);
        const uint32_t nb = min(64u, E - e0);
        for (uint32_t b = 0; b < nb; b++)
            if (U[static_cast<uint64_t>(e0 + b) * ld + j] > T(0)) bits |= 1ull << b;
        P[idx] = bits;
    }
}

// 8-bit length tables: LUT[(w*8 + byte)*256 + v] = sum of L over the set
// bits of v; grid.y = table when the lengths are per table.
template <typename T>
__global__ void build_lut_kernel(const T *__restrict__ len, uint32_t E, T *__restrict__ lut, uint64_t len_stride,
                                 uint64_t lut_stride) {
    const uint32_t wb = blockIdx.x;  // word * 8 + byte
    const uint32_t v = threadIdx.x;  // 0..255
    const uint32_t base = wb * 8;
    const T *L = len + blockIdx.y * len_stride;
    T s = T(0);
    for (uint32_t i = 0; i < 8; i++)
        if (((v >> i) & 1u) && base + i < E) s += L[base + i];
    lut[blockIdx.y * lut_stride + static_cast<uint64_t>(wb) * 256 + v] = s;
}

// Faith PD: per sample sum of L over non-root nodes with u > 0
// (src/unifrac.cpp:362-387), rows visited in postorder within fixed chunks.
static __global__ void faith_partial_kernel(const double *__restrict__ U, const double *__restrict__ len_by_row,
                                     const uint32_t *__restrict__ post_rows, uint32_t K, uint64_t ld,
                                     uint32_t chunk, double *__restrict__ partial) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    const uint32_t k0 = blockIdx.y * chunk;
    const uint32_t k1 = min(K, k0 + chunk);
    double s = 0.0;
    for (uint32_t k = k0; k < k1; k++) {
        const uint32_t row = post_rows[k];
        s += static_cast<double>(U[static_cast<uint64_t>(row) * ld + j] > 0.0) * len_by_row[row];
    }
    partial[static_cast<uint64_t>(blockIdx.y) * ld + j] = s;
}

// Diagonal of every table's full result (grid.y = table).
static __global__ void zero_diagonal_kernel(void *out, const TableDesc *__restrict__ tables, int fp64) {
    const TableDesc td = tables[blockIdx.y];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < td.n; k += gridDim.x * blockDim.x) {
        const uint64_t at = td.out_off + static_cast<uint64_t>(k) * td.n + k;
        if (fp64)
            static_cast<double *>(out)[at] = 0.0;
        else
            static_cast<float *>(out)[at] = 0.0f;
    }
}

// ---------------------------------------------------------- pair kernels

// Where a finished pair value goes.
struct OutSpec {
    int mode;  // 0 full n x n (T), 1 stripes [start, stop) x n (double), 2 condensed (double)
    void *ptr;
    uint32_t start, stop;
};

template <typename T>
__device__ __forceinline__ void emit_pair(const OutSpec &o, uint32_t n, uint32_t k, uint32_t l, T v) {
    if (k >= l || l >= n) return;
    if (o.mode == 0) {
        T *out = static_cast<T *>(o.ptr);
        out[static_cast<uint64_t>(k) * n + l] = v;
        out[static_cast<uint64_t>(l) * n + k] = v;
    } else if (o.mode == 1) {
        // pair (k, l) is stripe l-k-1 at position k and stripe n-(l-k)-1 at
        // position l (src/unifrac_cmp.cpp:54-96); the last stripe of an even n
        // holds every such pair twice
        double *out = static_cast<double *>(o.ptr);
        const uint32_t d = l - k;
        const uint32_t s1 = d - 1, s2 = n - d - 1;
        if (s1 >= o.start && s1 < o.stop) out[static_cast<uint64_t>(s1 - o.start) * n + k] = static_cast<double>(v);
        if (s2 >= o.start && s2 < o.stop) out[static_cast<uint64_t>(s2 - o.start) * n + l] = static_cast<double>(v);
    } else {
        // scipy condensed index (src/unifrac.cpp:99-120)
        double *out = static_cast<double *>(o.ptr);
        const uint64_t kk = k;
        out[kk * (2ull * n - kk - 1) / 2 + (l - k - 1)] = static_cast<double>(v);
    }
}

// Work of one pair launch: tiles (x = k block, y = l block in the group's
// columns, z = table) times node splits, walked by a persistent grid.
template <typename T>
struct PairArgs {
    const uint4 *tiles;
    uint32_t n_tiles;
    uint32_t n_splits;
    const TableDesc *tables;
    const T *U;       // embedding, or presence words for the bit kernels
    const T *C;       // raw counts (variance adjusted)
    const T *len;     // embedded lengths (table z at len + z * len_stride)
    uint64_t len_stride;
    const T *tot;     // per-sample totals in T (variance adjusted)
    const T *W;       // per-sample weighted sums (weighted normalized)
    const unsigned long long *P;  // presence words (unweighted)
    const T *lut;                 // 8-bit length tables (unweighted), table z at lut + z * lut_stride
    uint64_t lut_stride;
    uint32_t E;       // embedded rows (or words for the bit kernel)
    uint64_t ld;
    uint32_t rows_per_split;
    T alpha;
    OutSpec out;
    T *partial;       // per-split raw accumulators; nullptr when not split
    const int *tile_flags;  // when set, only tiles with a non-zero flag are computed
};

// ---- per-term operators (one (k, l) pair, one embedded node) -------------

template <typename T> __device__ __forceinline__ T tabs(T x) { return fabs(x); }

// src/unifrac_task_impl.hpp:107-193 (numerator |u-v| L)
template <typename T, bool NORMALIZED>
struct OpWeighted {
    static constexpr int NACC = 1;
    static constexpr bool COUNTS = false;
    __device__ static void term(T *acc, T a, T b, T, T, T, T L, T) { acc[0] = fma(tabs(a - b), L, acc[0]); }
    __device__ static T value(const T *acc, T wk, T wl) { return NORMALIZED ? acc[0] / (wk + wl) : acc[0]; }
};

// (u+v)^alpha for the general alpha kind.
template <typename T>
__device__ __forceinline__ T pow_alpha(T s, T alpha) {
    return pow(s, alpha);
}

// 1/sqrt(x): one rsqrt instead of a sqrt and a division.  Every term below is
// rewritten with it in a mathematically identical form (a few ulp per term).
template <typename T>
__device__ __forceinline__ T inv_sqrt(T x) {
    return rsqrt(x);
}

// src/unifrac_task_impl.hpp:924-1040: per node, with s = u + v and
// sp = s^alpha L, num += sp |u - v| / s and den += sp (nodes with s = 0 add
// nothing).  Alpha kinds: 1 (0.5) num += L |u-v| / sqrt(s), den += L sqrt(s);
// 2 (1) num += L |u-v|, den += L s; 3 (0) num += L |u-v| / s, den += L.
template <typename T, int AK>
struct OpGeneralized {
    static constexpr int NACC = 2;
    static constexpr bool COUNTS = false;
    __device__ static void term(T *acc, T a, T b, T, T, T, T L, T alpha) {
        const T s = a + b;
        if (s != T(0)) {
            if (AK == 2) {
                acc[0] = fma(L, tabs(a - b), acc[0]);
                acc[1] = fma(L, s, acc[1]);
            } else if (AK == 1) {
                const T t = L * inv_sqrt(s);
                acc[0] = fma(t, tabs(a - b), acc[0]);
                acc[1] = fma(t, s, acc[1]);
            } else if (AK == 3) {
                acc[0] = fma(L, tabs(a - b) / s, acc[0]);
                acc[1] += L;
            } else {
                const T sp = pow_alpha<T>(s, alpha) * L;
                acc[0] = fma(sp, tabs(a - b) / s, acc[0]);
                acc[1] += sp;
            }
        }
    }
    __device__ static T value(const T *acc, T, T) { return acc[0] / acc[1]; }
};

// src/unifrac_task_impl.hpp:435-502, 848-922: with vaw = sqrt(mi (m - mi)),
// num += |u - v| L / vaw and den += (u + v) L / vaw where vaw > 0.
template <typename T, bool NORMALIZED>
struct OpVawWeighted {
    static constexpr int NACC = NORMALIZED ? 2 : 1;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T) {
        const T mi = ca + cb;
        const T x = mi * (m - mi);
        if (x > T(0)) {
            const T t = L * inv_sqrt(x);
            acc[0] = fma(t, tabs(a - b), acc[0]);
            if (NORMALIZED) acc[1] = fma(t, a + b, acc[1]);
        }
    }
    __device__ static T value(const T *acc, T, T) { return NORMALIZED ? acc[0] / acc[NACC - 1] : acc[0]; }
};

// src/unifrac_task_impl.hpp:1042-1119: s1 = (u + v) / vaw, d1 = |u - v| / vaw,
// sp = s1^alpha L; num += sp d1 / s1, den += sp.
template <typename T, int AK>
struct OpVawGeneralized {
    static constexpr int NACC = 2;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T alpha) {
        const T mi = ca + cb;
        const T x = mi * (m - mi);
        if (x > T(0)) {
            const T r = inv_sqrt(x);
            const T s1 = (a + b) * r;
            const T d1 = tabs(a - b) * r;
            if (AK == 1) {
                const T t = L * inv_sqrt(s1);
                acc[0] = fma(t, d1, acc[0]);
                acc[1] = fma(t, s1, acc[1]);
            } else if (AK == 2) {
                acc[0] = fma(L, d1, acc[0]);
                acc[1] = fma(L, s1, acc[1]);
            } else if (AK == 3) {
                acc[0] = fma(L, d1 / s1, acc[0]);
                acc[1] += L;
            } else {
                const T sp = pow_alpha<T>(s1, alpha) * L;
                acc[0] = fma(sp, d1 / s1, acc[0]);
                acc[1] += sp;
            }
        }
    }
    __device__ static T value(const T *acc, T, T) { return acc[0] / acc[1]; }
};

// src/unifrac_task_impl.hpp:1755-1932: L / vaw where exactly one side is
// present (num) and where either is (den).
template <typename T, bool NORMALIZED>
struct OpVawUnweighted {
    static constexpr int NACC = NORMALIZED ? 2 : 1;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T) {
        const T mi = ca + cb;
        const T x = mi * (m - mi);
        if (x > T(0)) {
            const T lv = L * inv_sqrt(x);
            const bool pa = a > T(0), pb = b > T(0);
            if (pa != pb) acc[0] += lv;
            if (NORMALIZED && (pa || pb)) acc[1] += lv;
        }
    }
    __device__ static T value(const T *acc, T, T) { return NORMALIZED ? acc[0] / acc[NACC - 1] : acc[0]; }
};

// Unweighted over presence words (the 8-bit length-table form)
template <typename T, bool NORMALIZED>
struct OpUnweightedBits {
    static constexpr int NACC = NORMALIZED ? 2 : 1;
    __device__ static T value(const T *acc, T, T) { return NORMALIZED ? acc[0] / acc[NACC - 1] : acc[0]; }
};

// Single-precision sums over every embedded node run in two levels: each
// pipeline chunk (32 rows, or 4 presence words) is summed on its own and
// then added to the running total, so no fp32 sum grows over more than a few
// hundred terms in a row (the reference's GPU tasks likewise add one
// 112-node batch at a time into their stripes).
template <typename T>
constexpr bool kTwoLevel = sizeof(T) == 4;

// ---- tile geometry -------------------------------------------------------
// A thread owns TM rows (k) and TN columns (l) of the BM x BN tile, split in
// two halves (ty*TM/2 .. and BM/2 + ty*TM/2 ..) so each half is one vector
// load from shared memory.

template <int BM, int TM>
__device__ __forceinline__ int tile_row(int ty, int i) {
    return i < TM / 2 ? ty * (TM / 2) + i : BM / 2 + ty * (TM / 2) + (i - TM / 2);
}

template <typename T, int CNT>
__device__ __forceinline__ void load_half(T *dst, const T *src) {
    static_assert((CNT * sizeof(T)) % 16 == 0 || CNT * sizeof(T) == 8, "vector width");
    if constexpr (CNT * sizeof(T) == 8) {
        *reinterpret_cast<uint2 *>(dst) = *reinterpret_cast<const uint2 *>(src);
    } else {
#pragma unroll
        for (int q = 0; q < (CNT * (int)sizeof(T)) / 16; q++)
            reinterpret_cast<uint4 *>(dst)[q] = reinterpret_cast<const uint4 *>(src)[q];
    }
}

// Shared epilogue: per (i, j) owned by the thread, finish the value and emit
// it into the tile's table (W is indexed by group column, the output by the
// table's own sample index).
template <typename T, class Op, int BM, int BN, int TM, int TN>
__device__ __forceinline__ void pair_epilogue(const PairArgs<T> &a, const uint4 tile, int tx, int ty,
                                              const T (&acc)[TM][TN][Op::NACC]) {
    const TableDesc td = a.tables[tile.z];
    const uint32_t k0 = tile.x * BM, l0 = tile.y * BN;
    OutSpec o = a.out;
    if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const uint32_t kc = k0 + tile_row<BM, TM>(ty, i);
        const uint32_t k = kc - td.base;
        const T wk = (a.W && k < td.n) ? a.W[kc] : T(0);
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const uint32_t lc = l0 + tile_row<BN, TN>(tx, j);
            const uint32_t l = lc - td.base;
            if (k < l && l < td.n) {
                const T wl = a.W ? a.W[lc] : T(0);
                emit_pair<T>(o, td.n, k, l, Op::value(acc[i][j], wk, wl));
            }
        }
    }
}

template <typename T, class Op, int BM, int BN, int TM, int TN>
__device__ __forceinline__ void store_partial(const PairArgs<T> &a, uint32_t split, uint32_t tile,
                                              const T (&acc)[TM][TN][Op::NACC]) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NV = TM * TN * Op::NACC;
    T *base = a.partial + (static_cast<uint64_t>(split) * a.n_tiles + tile) * NV * NT;
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
            for (int c = 0; c < Op::NACC; c++)
                base[static_cast<uint64_t>((i * TN + j) * Op::NACC + c) * NT + threadIdx.x] = acc[i][j][c];
}

// Sum the per-split partials of each tile in split order, then emit.
template <typename T, class Op, int BM, int BN, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    split_finalize_kernel(const PairArgs<T> a, uint32_t n_splits) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NV = TM * TN * Op::NACC;
    constexpr int TX = BN / TN;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    T acc[TM][TN][Op::NACC];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
            for (int c = 0; c < Op::NACC; c++) acc[i][j][c] = T(0);
    for (uint32_t s = 0; s < n_splits; s++) {
        const T *base = a.partial + (static_cast<uint64_t>(s) * a.n_tiles + blockIdx.x) * NV * NT;
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++)
#pragma unroll
                for (int c = 0; c < Op::NACC; c++)
                    acc[i][j][c] += base[static_cast<uint64_t>((i * TN + j) * Op::NACC + c) * NT + threadIdx.x];
    }
    pair_epilogue<T, Op, BM, BN, TM, TN>(a, a.tiles[blockIdx.x], tx, ty, acc);
}

// ---- value pair kernel (weighted, generalized, variance adjusted) ---------
//
// Persistent grid over work items w = split * n_tiles + tile (split-major,
// so CTAs running together read the same node rows).  Each item streams its
// node rows through a two-stage cp.async pipeline of KC rows: BM values of the k block and BN
// of the l block per row (plus raw counts for variance adjustment) and the
// KC lengths.
template <typename T, class Op, int BM, int BN, int TM, int TN, int KC>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1) pair_values_kernel(const PairArgs<T> a) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int TX = BN / TN;
    constexpr int VEC = 16 / sizeof(T);
    constexpr int CPR_A = BM / VEC;  // 16-byte chunks per row
    constexpr int CPR_B = BN / VEC;
    constexpr bool CNT = Op::COUNTS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *As = reinterpret_cast<T *>(smem_raw);  // [2][KC][BM]
    T *Bs = As + 2 * KC * BM;                 // [2][KC][BN]
    T *Acs = Bs + 2 * KC * BN;                // [2][KC][BM] counts
    T *Bcs = Acs + (CNT ? 2 * KC * BM : 0);   // [2][KC][BN] counts
    T *Ls = Bcs + (CNT ? 2 * KC * BN : 0);    // [2][KC]

    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const uint32_t n_work = a.n_tiles * a.n_splits;
    for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
        const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
        if (a.tile_flags && !a.tile_flags[ti]) continue;  // uniform over the CTA
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * BM, l0 = tile.y * BN;
        const uint32_t e_begin = split * a.rows_per_split;
        const uint32_t e_end = min(a.E, e_begin + a.rows_per_split);
        const T *lenp = a.len + tile.z * a.len_stride;

        T acc[TM][TN][Op::NACC];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++)
#pragma unroll
                for (int c = 0; c < Op::NACC; c++) acc[i][j][c] = T(0);

        T tk[TM], tl[TN];
        if (CNT) {
#pragma unroll
            for (int i = 0; i < TM; i++) tk[i] = a.tot[k0 + tile_row<BM, TM>(ty, i)];
#pragma unroll
            for (int j = 0; j < TN; j++) tl[j] = a.tot[l0 + tile_row<BN, TN>(tx, j)];
        }

        auto load_stage = [&](int st, uint32_t e0) {
            for (int c = tid; c < KC * CPR_A; c += NT) {
                const int r = c / CPR_A, q = c % CPR_A;
                const uint32_t e = e0 + r;
                const bool ok = e < e_end;
                const uint64_t off = static_cast<uint64_t>(ok ? e : 0) * a.ld + k0 + q * VEC;
                cp_async16(As + (st * KC + r) * BM + q * VEC, a.U + off, ok ? 16 : 0);
                if (CNT) cp_async16(Acs + (st * KC + r) * BM + q * VEC, a.C + off, ok ? 16 : 0);
            }
            for (int c = tid; c < KC * CPR_B; c += NT) {
                const int r = c / CPR_B, q = c % CPR_B;
                const uint32_t e = e0 + r;
                const bool ok = e < e_end;
                const uint64_t off = static_cast<uint64_t>(ok ? e : 0) * a.ld + l0 + q * VEC;
                cp_async16(Bs + (st * KC + r) * BN + q * VEC, a.U + off, ok ? 16 : 0);
                if (CNT) cp_async16(Bcs + (st * KC + r) * BN + q * VEC, a.C + off, ok ? 16 : 0);
            }
            for (int c = tid; c < KC; c += NT) {
                const uint32_t e = e0 + c;
                const bool ok = e < e_end;
                cp_async_small<sizeof(T)>(Ls + st * KC + c, lenp + (ok ? e : 0), ok ? (int)sizeof(T) : 0);
            }
        };

        const uint32_t n_chunks = e_end > e_begin ? (e_end - e_begin + KC - 1) / KC : 0;
        if (n_chunks > 0) load_stage(0, e_begin);
        cp_async_commit();
        for (uint32_t ch = 0; ch < n_chunks; ch++) {
            const int st = ch & 1;
            if (ch + 1 < n_chunks) load_stage(st ^ 1, e_begin + (ch + 1) * KC);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            const T *as = As + st * KC * BM;
            const T *bs = Bs + st * KC * BN;
            const T *acs = Acs + st * KC * BM;
            const T *bcs = Bcs + st * KC * BN;
            auto chunk = [&](T (&dst)[TM][TN][Op::NACC]) {
#pragma unroll 2
                for (int c = 0; c < KC; c++) {
                    T av[TM], bv[TN], ac[TM], bc[TN];
                    load_half<T, TM / 2>(av, as + c * BM + ty * (TM / 2));
                    load_half<T, TM / 2>(av + TM / 2, as + c * BM + BM / 2 + ty * (TM / 2));
                    load_half<T, TN / 2>(bv, bs + c * BN + tx * (TN / 2));
                    load_half<T, TN / 2>(bv + TN / 2, bs + c * BN + BN / 2 + tx * (TN / 2));
                    if (CNT) {
                        load_half<T, TM / 2>(ac, acs + c * BM + ty * (TM / 2));
                        load_half<T, TM / 2>(ac + TM / 2, acs + c * BM + BM / 2 + ty * (TM / 2));
                        load_half<T, TN / 2>(bc, bcs + c * BN + tx * (TN / 2));
                        load_half<T, TN / 2>(bc + TN / 2, bcs + c * BN + BN / 2 + tx * (TN / 2));
                    }
                    const T L = Ls[st * KC + c];
#pragma unroll
                    for (int i = 0; i < TM; i++)
#pragma unroll
                        for (int j = 0; j < TN; j++)
                            Op::term(dst[i][j], av[i], bv[j], CNT ? ac[i] : T(0), CNT ? bc[j] : T(0),
                                     CNT ? tk[i] + tl[j] : T(0), L, a.alpha);
                }
            };
            if constexpr (kTwoLevel<T>) {
                // single precision: sum the chunk on its own, then fold it in
                T part[TM][TN][Op::NACC];
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++)
#pragma unroll
                        for (int q = 0; q < Op::NACC; q++) part[i][j][q] = T(0);
                chunk(part);
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++)
#pragma unroll
                        for (int q = 0; q < Op::NACC; q++) acc[i][j][q] += part[i][j][q];
            } else {
                chunk(acc);
            }
            __syncthreads();
        }
        cp_async_wait<0>();

        if (a.partial)
            store_partial<T, Op, BM, BN, TM, TN>(a, split, ti, acc);
        else
            pair_epilogue<T, Op, BM, BN, TM, TN>(a, tile, tx, ty, acc);
        __syncthreads();  // shared memory is reused by the next work item
    }
}

template <typename T, class Op, int BM, int BN, int KC>
constexpr size_t pair_values_smem() {
    return sizeof(T) * (2 * KC * (BM + BN) * (Op::COUNTS ? 2 : 1) + 2 * KC);
}

// ---- unweighted presence-word kernel ------------------------------------
//
// Per 64-node word: xor / or of the two samples' presence bits, then the sum
// of the 8 byte-indexed length tables (src/unifrac_task_impl.hpp:1193-1278).
// KW words per pipeline stage: BM + BN presence words and KW*2048 table
// entries.
template <typename T, bool NORMALIZED, int BM, int BN, int TM, int TN, int KW>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1) pair_bits_kernel(const PairArgs<T> a) {
    using Op = OpUnweightedBits<T, NORMALIZED>;
    using u64 = unsigned long long;
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int TX = BN / TN;
    constexpr int LUTW = 8 * 256;
    constexpr int LUT_CHUNKS = LUTW * sizeof(T) / 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ls = reinterpret_cast<T *>(smem_raw);             // [2][KW][2048]
    u64 *As = reinterpret_cast<u64 *>(Ls + 2 * KW * LUTW);  // [2][KW][BM]
    u64 *Bs = As + 2 * KW * BM;                             // [2][KW][BN]

    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const uint32_t n_work = a.n_tiles * a.n_splits;
    for (uint32_t wi = blockIdx.x; wi < n_work; wi += gridDim.x) {
        const uint32_t split = wi / a.n_tiles, ti = wi - split * a.n_tiles;
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * BM, l0 = tile.y * BN;
        const uint32_t w_begin = split * a.rows_per_split;
        const uint32_t w_end = min(a.E, w_begin + a.rows_per_split);
        const T *lutp = a.lut + tile.z * a.lut_stride;

        T acc[TM][TN][Op::NACC];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++)
#pragma unroll
                for (int c = 0; c < Op::NACC; c++) acc[i][j][c] = T(0);

        auto load_stage = [&](int st, uint32_t w0) {
            for (int c = tid; c < KW * LUT_CHUNKS; c += NT) {
                const int r = c / LUT_CHUNKS, q = c % LUT_CHUNKS;
                const uint32_t w = w0 + r;
                const bool ok = w < w_end;
                cp_async16(reinterpret_cast<unsigned char *>(Ls + (st * KW + r) * LUTW) + q * 16,
                           reinterpret_cast<const unsigned char *>(lutp + static_cast<uint64_t>(ok ? w : 0) * LUTW) +
                               q * 16,
                           ok ? 16 : 0);
            }
            for (int c = tid; c < KW * (BM / 2); c += NT) {
                const int r = c / (BM / 2), q = c % (BM / 2);
                const uint32_t w = w0 + r;
                const bool ok = w < w_end;
                cp_async16(As + (st * KW + r) * BM + q * 2, a.P + static_cast<uint64_t>(ok ? w : 0) * a.ld + k0 + q * 2,
                           ok ? 16 : 0);
            }
            for (int c = tid; c < KW * (BN / 2); c += NT) {
                const int r = c / (BN / 2), q = c % (BN / 2);
                const uint32_t w = w0 + r;
                const bool ok = w < w_end;
                cp_async16(Bs + (st * KW + r) * BN + q * 2, a.P + static_cast<uint64_t>(ok ? w : 0) * a.ld + l0 + q * 2,
                           ok ? 16 : 0);
            }
        };

        const uint32_t n_chunks = w_end > w_begin ? (w_end - w_begin + KW - 1) / KW : 0;
        if (n_chunks > 0) load_stage(0, w_begin);
        cp_async_commit();
        for (uint32_t ch = 0; ch < n_chunks; ch++) {
            const int st = ch & 1;
            if (ch + 1 < n_chunks) load_stage(st ^ 1, w_begin + (ch + 1) * KW);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            T part[TM][TN][Op::NACC];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++)
#pragma unroll
                    for (int q = 0; q < Op::NACC; q++) part[i][j][q] = T(0);
            T(&dst)[TM][TN][Op::NACC] = kTwoLevel<T> ? part : acc;
            for (int r = 0; r < KW; r++) {
                const T *lut = Ls + (st * KW + r) * LUTW;
                const u64 *as = As + (st * KW + r) * BM;
                const u64 *bs = Bs + (st * KW + r) * BN;
                u64 av[TM], bv[TN];
#pragma unroll
                for (int i = 0; i < TM; i++) av[i] = as[tile_row<BM, TM>(ty, i)];
#pragma unroll
                for (int j = 0; j < TN; j++) bv[j] = bs[tile_row<BN, TN>(tx, j)];
#pragma unroll
                for (int i = 0; i < TM; i++) {
#pragma unroll
                    for (int j = 0; j < TN; j++) {
                        const u64 o = av[i] | bv[j];
                        if (o == 0ull) continue;
                        const u64 x = av[i] ^ bv[j];
                        const uint32_t xl = static_cast<uint32_t>(x), xh = static_cast<uint32_t>(x >> 32);
                        dst[i][j][0] += lut[xl & 255u] + lut[256 + ((xl >> 8) & 255u)] + lut[512 + ((xl >> 16) & 255u)] +
                                        lut[768 + (xl >> 24)] + lut[1024 + (xh & 255u)] +
                                        lut[1280 + ((xh >> 8) & 255u)] + lut[1536 + ((xh >> 16) & 255u)] +
                                        lut[1792 + (xh >> 24)];
                        if (NORMALIZED) {
                            const uint32_t ol = static_cast<uint32_t>(o), oh = static_cast<uint32_t>(o >> 32);
                            dst[i][j][1] += lut[ol & 255u] + lut[256 + ((ol >> 8) & 255u)] +
                                            lut[512 + ((ol >> 16) & 255u)] + lut[768 + (ol >> 24)] +
                                            lut[1024 + (oh & 255u)] + lut[1280 + ((oh >> 8) & 255u)] +
                                            lut[1536 + ((oh >> 16) & 255u)] + lut[1792 + (oh >> 24)];
                        }
                    }
                }
            }
            if constexpr (kTwoLevel<T>) {
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++)
#pragma unroll
                        for (int q = 0; q < Op::NACC; q++) acc[i][j][q] += part[i][j][q];
            }
            __syncthreads();
        }
        cp_async_wait<0>();

        if (a.partial)
            store_partial<T, Op, BM, BN, TM, TN>(a, split, ti, acc);
        else
            pair_epilogue<T, Op, BM, BN, TM, TN>(a, tile, tx, ty, acc);
        __syncthreads();  // shared memory is reused by the next work item
    }
}

template <typename T, int BM, int BN, int KW>
constexpr size_t pair_bits_smem() {
    return 2 * KW * (8 * 256 * sizeof(T) + (BM + BN) * sizeof(unsigned long long));
}

}  // namespace dev
}  // namespace ssu
