// CUDA kernels of the B200 UniFrac engine (sm_100a).
//
// Data layout in HBM (one table):
//   U[row][j]   proportion embedding, rows = non-root nodes (embedded rows
//               first, in postorder), j = sample; row stride `ld` = n rounded
//               up to 128 so every tile load is in bounds and 16-byte aligned;
//               padding columns are zero.
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

// --------------------------------------------------------------- embedding

// Tip rows: zero the row, then scatter the tip's CSR entries; proportions
// are data / total in fp64 and then rounded to T (src/biom_inmem.cpp:473-497).
template <typename T, bool COUNTS>
__global__ void embed_tips_kernel(const uint32_t *__restrict__ tip_rows, const int32_t *__restrict__ tip_obs,
                                  uint32_t n_tips, const uint32_t *__restrict__ indptr,
                                  const uint32_t *__restrict__ indices, const double *__restrict__ data,
                                  const double *__restrict__ totals, bool normalize, T *__restrict__ U,
                                  T *__restrict__ C, uint64_t ld) {
    for (uint32_t t = blockIdx.x; t < n_tips; t += gridDim.x) {
        const uint64_t row = tip_rows[t];
        T *u = U + row * ld;
        T *c = COUNTS ? C + row * ld : nullptr;
        for (uint64_t j = threadIdx.x; j < ld; j += blockDim.x) {
            u[j] = T(0);
            if (COUNTS) c[j] = T(0);
        }
        __syncthreads();
        const int32_t r = tip_obs[t];
        if (r >= 0) {
            for (uint32_t q = indptr[r] + threadIdx.x; q < indptr[r + 1]; q += blockDim.x) {
                const uint32_t j = indices[q];
                const double v = data[q];
                u[j] = normalize ? static_cast<T>(v / totals[j]) : static_cast<T>(v);
                if (COUNTS) c[j] = static_cast<T>(v);
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
                                   T *__restrict__ U, T *__restrict__ C, uint64_t ld, uint32_t col_blocks) {
    using V = typename Vec16<T>::type;
    const uint64_t nvec = ld / Vec16<T>::n;
    const uint64_t total = static_cast<uint64_t>(n_rows) * col_blocks;
    for (uint64_t b = blockIdx.x; b < total; b += gridDim.x) {
        const uint32_t row = rows[b / col_blocks];
        const uint64_t v = (b % col_blocks) * blockDim.x + threadIdx.x;
        if (v >= nvec) continue;
        V s = Vec16<T>::zero();
        V sc = Vec16<T>::zero();
        for (uint32_t c = child_ptr[row]; c < child_ptr[row + 1]; c++) {
            const uint64_t cr = child_rows[c];
            s = Vec16<T>::add(s, reinterpret_cast<const V *>(U + cr * ld)[v]);
            if (COUNTS) sc = Vec16<T>::add(sc, reinterpret_cast<const V *>(C + cr * ld)[v]);
        }
        reinterpret_cast<V *>(U + static_cast<uint64_t>(row) * ld)[v] = s;
        if (COUNTS) reinterpret_cast<V *>(C + static_cast<uint64_t>(row) * ld)[v] = sc;
    }
}

// W[j] = sum_e L_e u_e[j] over embedded rows, in fixed row chunks (partial
// sums, then an in-order reduction), the one-sided sums of
// src/unifrac_task_impl.hpp:51-103.
template <typename T>
__global__ void weighted_sums_partial_kernel(const T *__restrict__ U, const T *__restrict__ len, uint32_t E,
                                             uint64_t ld, uint32_t chunk, T *__restrict__ partial) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    const uint32_t e0 = blockIdx.y * chunk;
    const uint32_t e1 = min(E, e0 + chunk);
    T s = T(0);
    for (uint32_t e = e0; e < e1; e++) s = fma(U[static_cast<uint64_t>(e) * ld + j], len[e], s);
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

// 8-bit length tables: LUT[(w*8 + byte)*256 + v] = sum of L over the set bits of v.
template <typename T>
__global__ void build_lut_kernel(const T *__restrict__ len, uint32_t E, T *__restrict__ lut) {
    const uint32_t wb = blockIdx.x;  // word * 8 + byte
    const uint32_t v = threadIdx.x;  // 0..255
    const uint32_t base = wb * 8;
    T s = T(0);
    for (uint32_t i = 0; i < 8; i++)
        if (((v >> i) & 1u) && base + i < E) s += len[base + i];
    lut[static_cast<uint64_t>(wb) * 256 + v] = s;
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

static __global__ void zero_diagonal_kernel(void *out, uint32_t n, int fp64) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (fp64)
        static_cast<double *>(out)[static_cast<uint64_t>(k) * n + k] = 0.0;
    else
        static_cast<float *>(out)[static_cast<uint64_t>(k) * n + k] = 0.0f;
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

template <typename T>
struct PairArgs {
    const uint2 *tiles;
    uint32_t n_tiles;
    const T *U;       // embedding, or presence words for the bit kernels
    const T *C;       // raw counts (variance adjusted)
    const T *len;     // embedded lengths
    const T *tot;     // per-sample totals in T (variance adjusted)
    const T *W;       // per-sample weighted sums (weighted normalized)
    const unsigned long long *P;  // presence words (unweighted)
    const T *lut;                 // 8-bit length tables (unweighted)
    uint32_t E;       // embedded rows (or words for the bit kernel)
    uint64_t ld;
    uint32_t n;
    uint32_t rows_per_split;
    T alpha;
    OutSpec out;
    T *partial;       // per-split raw accumulators; nullptr when not split
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

// (u+v)^alpha with the exact special cases: alpha 1 and 0 are exact in C's
// pow, and a correctly rounded pow(x, 0.5) is the correctly rounded sqrt.
template <typename T, int AK>
__device__ __forceinline__ T pow_alpha(T s, T alpha) {
    if (AK == 1) return sqrt(s);
    if (AK == 2) return s;
    if (AK == 3) return T(1);
    return pow(s, alpha);
}

// src/unifrac_task_impl.hpp:924-1040
template <typename T, int AK>
struct OpGeneralized {
    static constexpr int NACC = 2;
    static constexpr bool COUNTS = false;
    __device__ static void term(T *acc, T a, T b, T, T, T, T L, T alpha) {
        const T s = a + b;
        if (s != T(0)) {
            const T sp = pow_alpha<T, AK>(s, alpha) * L;
            acc[0] = fma(sp, tabs(a - b) / s, acc[0]);
            acc[1] += sp;
        }
    }
    __device__ static T value(const T *acc, T, T) { return acc[0] / acc[1]; }
};

// src/unifrac_task_impl.hpp:435-502, 848-922
template <typename T, bool NORMALIZED>
struct OpVawWeighted {
    static constexpr int NACC = NORMALIZED ? 2 : 1;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T) {
        const T mi = ca + cb;
        const T vaw = sqrt(mi * (m - mi));
        if (vaw > T(0)) {
            acc[0] += (tabs(a - b) * L) / vaw;
            if (NORMALIZED) acc[1] += ((a + b) * L) / vaw;
        }
    }
    __device__ static T value(const T *acc, T, T) { return NORMALIZED ? acc[0] / acc[NACC - 1] : acc[0]; }
};

// src/unifrac_task_impl.hpp:1042-1119
template <typename T, int AK>
struct OpVawGeneralized {
    static constexpr int NACC = 2;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T alpha) {
        const T mi = ca + cb;
        const T vaw = sqrt(mi * (m - mi));
        if (vaw > T(0)) {
            const T s1 = (a + b) / vaw;
            const T d1 = tabs(a - b) / vaw;
            const T sp = pow_alpha<T, AK>(s1, alpha) * L;
            acc[0] = fma(sp, d1 / s1, acc[0]);
            acc[1] += sp;
        }
    }
    __device__ static T value(const T *acc, T, T) { return acc[0] / acc[1]; }
};

// src/unifrac_task_impl.hpp:1755-1932
template <typename T, bool NORMALIZED>
struct OpVawUnweighted {
    static constexpr int NACC = NORMALIZED ? 2 : 1;
    static constexpr bool COUNTS = true;
    __device__ static void term(T *acc, T a, T b, T ca, T cb, T m, T L, T) {
        const T mi = ca + cb;
        const T vaw = sqrt(mi * (m - mi));
        if (vaw > T(0)) {
            const T lv = L / vaw;
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

// Shared epilogue: per (i, j) owned by the thread, finish the value and emit it.
template <typename T, class Op, int BM, int BN, int TM, int TN>
__device__ __forceinline__ void pair_epilogue(const PairArgs<T> &a, uint32_t k0, uint32_t l0, int tx, int ty,
                                              const T (&acc)[TM][TN][Op::NACC]) {
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const uint32_t k = k0 + tile_row<BM, TM>(ty, i);
        const T wk = (a.W && k < a.n) ? a.W[k] : T(0);
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const uint32_t l = l0 + tile_row<BN, TN>(tx, j);
            if (k < l && l < a.n) {
                const T wl = a.W ? a.W[l] : T(0);
                emit_pair<T>(a.out, a.n, k, l, Op::value(acc[i][j], wk, wl));
            }
        }
    }
}

template <typename T, class Op, int BM, int BN, int TM, int TN>
__device__ __forceinline__ void store_partial(const PairArgs<T> &a, const T (&acc)[TM][TN][Op::NACC]) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NV = TM * TN * Op::NACC;
    T *base = a.partial + (static_cast<uint64_t>(blockIdx.y) * a.n_tiles + blockIdx.x) * NV * NT;
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
    const uint2 tile = a.tiles[blockIdx.x];
    pair_epilogue<T, Op, BM, BN, TM, TN>(a, tile.x * BM, tile.y * BN, tx, ty, acc);
}

// ---- value pair kernel (weighted, generalized, variance adjusted) ---------
//
// Grid: x = tile, y = node split.  Each CTA streams its node rows through a
// two-stage cp.async pipeline of KC rows: BM values of the k block and BN
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

    const uint2 tile = a.tiles[blockIdx.x];
    const uint32_t k0 = tile.x * BM, l0 = tile.y * BN;
    const uint32_t e_begin = blockIdx.y * a.rows_per_split;
    const uint32_t e_end = min(a.E, e_begin + a.rows_per_split);
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;

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
            cp_async_small<sizeof(T)>(Ls + st * KC + c, a.len + (ok ? e : 0), ok ? (int)sizeof(T) : 0);
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
                    Op::term(acc[i][j], av[i], bv[j], CNT ? ac[i] : T(0), CNT ? bc[j] : T(0),
                             CNT ? tk[i] + tl[j] : T(0), L, a.alpha);
        }
        __syncthreads();
    }
    cp_async_wait<0>();

    if (a.partial)
        store_partial<T, Op, BM, BN, TM, TN>(a, acc);
    else
        pair_epilogue<T, Op, BM, BN, TM, TN>(a, k0, l0, tx, ty, acc);
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

    const uint2 tile = a.tiles[blockIdx.x];
    const uint32_t k0 = tile.x * BM, l0 = tile.y * BN;
    const uint32_t w_begin = blockIdx.y * a.rows_per_split;
    const uint32_t w_end = min(a.E, w_begin + a.rows_per_split);
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;

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
                       reinterpret_cast<const unsigned char *>(a.lut + static_cast<uint64_t>(ok ? w : 0) * LUTW) +
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
                    acc[i][j][0] += lut[xl & 255u] + lut[256 + ((xl >> 8) & 255u)] + lut[512 + ((xl >> 16) & 255u)] +
                                    lut[768 + (xl >> 24)] + lut[1024 + (xh & 255u)] +
                                    lut[1280 + ((xh >> 8) & 255u)] + lut[1536 + ((xh >> 16) & 255u)] +
                                    lut[1792 + (xh >> 24)];
                    if (NORMALIZED) {
                        const uint32_t ol = static_cast<uint32_t>(o), oh = static_cast<uint32_t>(o >> 32);
                        acc[i][j][1] += lut[ol & 255u] + lut[256 + ((ol >> 8) & 255u)] +
                                        lut[512 + ((ol >> 16) & 255u)] + lut[768 + (ol >> 24)] +
                                        lut[1024 + (oh & 255u)] + lut[1280 + ((oh >> 8) & 255u)] +
                                        lut[1536 + ((oh >> 16) & 255u)] + lut[1792 + (oh >> 24)];
                    }
                }
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();

    if (a.partial)
        store_partial<T, Op, BM, BN, TM, TN>(a, acc);
    else
        pair_epilogue<T, Op, BM, BN, TM, TN>(a, k0, l0, tx, ty, acc);
}

template <typename T, int BM, int BN, int KW>
constexpr size_t pair_bits_smem() {
    return 2 * KW * (8 * 256 * sizeof(T) + (BM + BN) * sizeof(unsigned long long));
}

}  // namespace dev
}  // namespace ssu
